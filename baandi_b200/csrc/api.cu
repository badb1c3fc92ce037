// C ABI of libbaandi_b200.so: contexts, operators (tables in HBM, stick plan, FFT
// plans, nonlocal operands) and the apply entry points.  See include/baandi_gpu.h.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "gemm_tc.cuh"
#include "op_internal.h"

namespace bg {
static thread_local std::string g_error;
void set_global_error(const std::string& msg) { g_error = msg; }
std::string global_error() { return g_error; }
}  // namespace bg

using namespace bg;

namespace bg {
int fail(bg_ctx* ctx, int code, const std::string& msg) {
  if (ctx) {
    ctx->error = msg;
  } else {
    set_global_error(msg);
  }
  return code;
}

int cuda_fail(bg_ctx* ctx, cudaError_t e, const char* what) {
  return fail(ctx, BG_EDEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace bg

namespace {

template <class T>
int upload(bg_op* op, const T* host, size_t count, T** out) {
  auto b = std::make_unique<DevBuf>();
  b->bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&b->p, b->bytes);
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "cudaMalloc");
  if (count && host) {
    e = cudaMemcpy(b->p, host, count * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(op->ctx, e, "cudaMemcpy");
  }
  *out = static_cast<T*>(b->p);
  op->bufs.push_back(std::move(b));
  return BG_OK;
}

int alloc(bg_op* op, size_t bytes, void** out, DevBuf** keep = nullptr) {
  auto b = std::make_unique<DevBuf>();
  b->bytes = std::max<size_t>(bytes, 16);
  cudaError_t e = cudaMalloc(&b->p, b->bytes);
  if (e != cudaSuccess) return fail(op->ctx, BG_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  *out = b->p;
  if (keep) *keep = b.get();
  op->bufs.push_back(std::move(b));
  return BG_OK;
}

// Host-buffer chunks of bg_kset_apply: about an eighth of the call's x per chunk, within
// these bounds (enough chunks to overlap, few enough launches).
constexpr size_t kChunkMin = (size_t)4 << 20, kChunkMax = (size_t)64 << 20;

// A host pointer the driver would stage itself (not page-locked or registered).
bool host_is_pageable(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeUnregistered;
}

// memcpy split over the host threads (pageable <-> pinned staging).
void parallel_copy(void* dst, const void* src, size_t bytes) {
  const int nt = bytes < ((size_t)4 << 20) ? 1 : std::min(16, std::max(1, omp_get_max_threads()));
  if (nt == 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t per = ((bytes + nt - 1) / nt + 4095) / 4096 * 4096;
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int t = 0; t < nt; ++t) {
    const size_t o = (size_t)t * per;
    if (o < bytes) std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, std::min(per, bytes - o));
  }
}

}  // namespace

namespace bg {
bool make_fft_plan(int n, FftPlan* p) {
  if (n < 1 || n > 128) return false;
  p->n = n;
  p->nst = 0;
  int m = n;
  for (int r : {4, 2, 3, 5}) {
    while (m % r == 0) {
      if (p->nst == kMaxStages) return false;
      p->radix[p->nst++] = r;
      m /= r;
    }
  }
  if (m != 1) return false;
  for (int s = 0; s < p->nst; ++s)
    if (n / p->radix[s] > 32 * kButterfliesPerLane) return false;
  return true;
}

std::vector<double> twiddles(int n) {
  std::vector<double> t(2 * n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int q = 0; q < n; ++q) {
    const long double a = two_pi * (long double)q / (long double)n;
    t[2 * q] = (double)cosl(a);
    t[2 * q + 1] = (double)sinl(a);
  }
  return t;
}
}  // namespace bg

namespace {

// Split of the P^H X reduction over rows: enough (tile, split) blocks for about eight
// 64-thread tile blocks per SM (148 SMs), chunks a multiple of 32 rows.
// Row splits of the projection P^H X over `tiles` 48 x 48 output tiles (k_project: 256
// threads, two blocks per SM): the smallest count whose blocks fill at least 85 % of
// whole waves of 2 x 148 blocks, at least 128 rows per split; kchunk = rows per split.
int ksplit_tiles(int64_t rows, int64_t tiles, int* kchunk, int64_t ks_cap = 1 << 30) {
  const int64_t slots = 2 * 148;
  const int64_t max_ks = std::max<int64_t>(1, std::min<int64_t>({64, (rows + 127) / 128, ks_cap}));
  int64_t ks = 1;
  double best = 0.0;
  for (int64_t k = 1; k <= max_ks; ++k) {
    const int64_t blocks = tiles * k, waves = (blocks + slots - 1) / slots;
    const double eff = (double)blocks / (double)(waves * slots);
    if (eff > best + 1e-9) {
      best = eff;
      ks = k;
    }
    if (eff >= 0.85) break;
  }
  int64_t chunk = (rows + ks - 1) / ks;
  chunk = ((chunk + 31) / 32) * 32;
  ks = (rows + chunk - 1) / chunk;
  *kchunk = (int)chunk;
  return (int)ks;
}

int ksplit_for(int64_t rows, int nproj, int64_t cols, int* kchunk) {
  return ksplit_tiles(rows, (int64_t)((nproj + 47) / 48) * ((cols + 47) / 48), kchunk);
}

// Build the stick plan, the tables and the nonlocal operands of one operator.
int build_op(bg_ctx* ctx, const bg_basis_desc* b, const bg_projectors* pr, int64_t capacity, bool gamma,
             bg_op** out) {
  if (!ctx || !b || !out || !b->miller || !b->kinetic) return fail(ctx, BG_EINVAL, "null argument");
  if (b->npw < 1 || capacity < 1 || capacity > 65535) return fail(ctx, BG_ESHAPE, "npw/capacity out of range");
  for (int i = 0; i < 3; ++i)
    if (b->dims[i] < 1) return fail(ctx, BG_ESHAPE, "grid dimensions");
  const int64_t npw = b->npw;
  for (int64_t g = 0; g < npw; ++g)
    if (!std::isfinite(b->kinetic[g])) return fail(ctx, BG_ENONFINITE, "kinetic diagonal not finite");
  int nproj = pr ? pr->nproj : 0;
  if (nproj < 0 || (nproj > 0 && (!pr->table || !pr->channels || !pr->couplings)))
    return fail(ctx, BG_EINVAL, "projector arguments");
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaSetDevice");

  auto op = std::make_unique<bg_op>();
  op->ctx = ctx;
  op->gamma = gamma;
  op->rows = npw;
  op->cap = capacity;
  op->cap_units = gamma ? (capacity + 1) / 2 : capacity;
  for (int i = 0; i < 3; ++i) op->dims[i] = b->dims[i];
  const int n0 = b->dims[0], n1 = b->dims[1], n2 = b->dims[2];

  // FFT index of every row
  std::vector<int64_t> flat(npw);
  const int dims[3] = {n0, n1, n2};
  if (fft_index(b->miller, npw, dims, b->gamma != 0 || gamma, flat.data()) != BG_OK)
    return fail(ctx, BG_ESHAPE, "Miller index outside the FFT grid or two rows on one grid point");

  // Gamma mirror maps
  std::vector<int64_t> plus, minus;
  if (gamma) {
    if (half_sphere(b->miller, npw, &plus, &minus) != BG_OK)
      return fail(ctx, BG_ESHAPE, "basis is not an inversion-symmetric Gamma sphere with G=0 first");
  }

  // sticks: (x, y) lines along z; a stick and its mirror adjacent
  std::map<int64_t, int> stick_id;  // x*n1+y -> provisional
  for (int64_t g = 0; g < npw; ++g) stick_id[flat[g] / n2] = 0;
  std::vector<int64_t> keys;
  for (auto& kv : stick_id) keys.push_back(kv.first);
  std::vector<char> used(keys.size(), 0);
  std::map<int64_t, size_t> key_index;
  for (size_t i = 0; i < keys.size(); ++i) key_index[keys[i]] = i;
  std::vector<std::vector<int64_t>> units;  // groups of 1 or 2 sticks that must stay together
  for (size_t i = 0; i < keys.size(); ++i) {
    if (used[i]) continue;
    used[i] = 1;
    const int64_t x = keys[i] / n1, y = keys[i] % n1;
    const int64_t mk = ((n0 - x) % n0) * n1 + (n1 - y) % n1;
    auto it = key_index.find(mk);
    if (it != key_index.end() && !used[it->second]) {
      used[it->second] = 1;
      units.push_back({keys[i], mk});
    } else {
      units.push_back({keys[i]});
    }
  }
  const int sg = 32;
  std::vector<int> grp_stick{0};
  std::vector<int64_t> order;  // stick -> key
  for (auto& u : units) {
    const int cur = (int)order.size() - grp_stick.back();
    if (cur + (int)u.size() > sg) grp_stick.push_back((int)order.size());
    for (int64_t k : u) order.push_back(k);
  }
  grp_stick.push_back((int)order.size());
  const int S = (int)order.size();
  const int ngroups = (int)grp_stick.size() - 1;
  std::vector<int> stick_of_key_group(S), group_of_stick(S);
  std::map<int64_t, int> stick_of_key;
  for (int s = 0; s < S; ++s) stick_of_key[order[s]] = s;
  for (int gi = 0; gi < ngroups; ++gi)
    for (int s = grp_stick[gi]; s < grp_stick[gi + 1]; ++s) group_of_stick[s] = gi;

  BoxGeo& G = op->g;
  G.n0 = n0;
  G.n1 = n1;
  G.n2 = n2;
  G.ld2 = n2 | 1;
  G.pitch = n1 | 1;
  G.sg = sg;
  G.vstride = (n0 * n1 + 1) & ~1;
  G.vstridef = (n0 * n1 + 3) & ~3;
  G.inv_n = 1.0 / ((double)n0 * n1 * n2);
  if (!make_fft_plan(n0, &G.p0) || !make_fft_plan(n1, &G.p1) || !make_fft_plan(n2, &G.p2))
    return fail(ctx, BG_ESHAPE, "grid length must be 2,3,5-smooth and at most 128");

  // position of every row in its group's shared-memory lines
  auto pos_of = [&](int64_t g, int* group) {
    const int s = stick_of_key[flat[g] / n2];
    *group = group_of_stick[s];
    return (s - grp_stick[*group]) * G.ld2 + (int)(flat[g] % n2);
  };
  std::vector<std::vector<std::pair<int, int>>> per_group(ngroups);
  std::vector<int> code(npw, 0);
  if (gamma) {
    for (size_t i = 1; i < plus.size(); ++i) {
      code[plus[i]] = (int)(2 * i - 1);
      code[minus[i]] = -(int)(2 * i - 1);
    }
  }
  for (int64_t g = 0; g < npw; ++g) {
    int grp;
    const int p = pos_of(g, &grp);
    per_group[grp].push_back({gamma ? code[g] : (int)g, p});
  }
  std::vector<int> grp_entry{0};
  std::vector<int> entries;
  for (int gi = 0; gi < ngroups; ++gi) {
    for (auto& e : per_group[gi]) {
      entries.push_back(e.first);
      entries.push_back(e.second);
    }
    grp_entry.push_back((int)(entries.size() / 2));
  }
  std::vector<int> grp_rep{0}, reps;
  if (gamma) {
    std::vector<std::vector<std::array<int, 4>>> rg(ngroups);
    for (size_t i = 0; i < plus.size(); ++i) {
      int ga, gb;
      const int pp = pos_of(plus[i], &ga);
      const int pm = pos_of(minus[i], &gb);
      if (ga != gb) return fail(ctx, BG_ESHAPE, "internal: mirror split across stick groups");
      rg[ga].push_back({i == 0 ? 0 : (int)(2 * i - 1), pp, pm, 0});
    }
    for (int gi = 0; gi < ngroups; ++gi) {
      for (auto& r : rg[gi]) reps.insert(reps.end(), r.begin(), r.end());
      grp_rep.push_back((int)(reps.size() / 4));
    }
  }
  std::vector<int> stick_plane(S), xact, line_stick;
  unsigned xbits[4] = {0u, 0u, 0u, 0u};
  {
    std::vector<char> xs(n0, 0);
    std::vector<int> at((size_t)n0 * n1, -1);
    for (int s = 0; s < S; ++s) {
      const int x = (int)(order[s] / n1), y = (int)(order[s] % n1);
      stick_plane[s] = x * G.pitch + y;
      at[(size_t)x * n1 + y] = s;
      xs[x] = 1;
    }
    for (int x = 0; x < n0; ++x)
      if (xs[x]) {
        xact.push_back(x);
        line_stick.insert(line_stick.end(), at.begin() + (size_t)x * n1, at.begin() + (size_t)(x + 1) * n1);
        xbits[x >> 5] |= 1u << (x & 31);
      }
  }

  // kinetic in row order (Gamma: ORC order, each pair row carries its representative's value)
  std::vector<double> kin(npw);
  if (gamma) {
    kin[0] = b->kinetic[0];
    for (size_t i = 1; i < plus.size(); ++i) kin[2 * i - 1] = kin[2 * i] = b->kinetic[plus[i]];
  } else {
    std::copy(b->kinetic, b->kinetic + npw, kin.begin());
  }

  OpTables& T = op->t;
  T.gamma = gamma ? 1 : 0;
  T.rows = (int)npw;
  T.S = S;
  T.ngroups = ngroups;
  T.nxact = (int)xact.size();
  T.yper = plane_lines_per_warp(n0, n1, T.nxact);
  T.yper16 = plane_lines_per_warp(n0, n1, T.nxact, 16);
  int rc;
  int* d_int;
  if ((rc = upload(op.get(), grp_stick.data(), grp_stick.size(), &d_int))) return rc;
  T.grp_stick = d_int;
  if ((rc = upload(op.get(), grp_entry.data(), grp_entry.size(), &d_int))) return rc;
  T.grp_entry = d_int;
  if ((rc = upload(op.get(), entries.data(), entries.size(), &d_int))) return rc;
  T.entries = reinterpret_cast<const int2*>(d_int);
  if (gamma) {
    if ((rc = upload(op.get(), grp_rep.data(), grp_rep.size(), &d_int))) return rc;
    T.grp_rep = d_int;
    if ((rc = upload(op.get(), reps.data(), reps.size(), &d_int))) return rc;
    T.reps = reinterpret_cast<const int4*>(d_int);
  }
  if ((rc = upload(op.get(), stick_plane.data(), stick_plane.size(), &d_int))) return rc;
  T.stick_plane = d_int;
  if ((rc = upload(op.get(), xact.data(), xact.size(), &d_int))) return rc;
  T.xact = d_int;
  if ((rc = upload(op.get(), line_stick.data(), line_stick.size(), &d_int))) return rc;
  T.line_stick = d_int;
  for (int w = 0; w < 4; ++w) T.xbits[w] = xbits[w];
  double* d_dbl;
  if ((rc = upload(op.get(), kin.data(), kin.size(), &d_dbl))) return rc;
  T.kinetic = d_dbl;
  std::vector<double> nanv((size_t)G.vstride * n2, std::nan(""));
  if ((rc = upload(op.get(), nanv.data(), nanv.size(), &d_dbl))) return rc;
  T.vt = d_dbl;
  std::vector<float> nanf((size_t)G.vstridef * n2, std::nanf(""));
  float* d_flt;
  if ((rc = upload(op.get(), nanf.data(), nanf.size(), &d_flt))) return rc;
  T.vtf = d_flt;
  void* vp;
  if ((rc = alloc(op.get(), sizeof(double2) * (size_t)op->cap_units * n2 * S, &vp))) return rc;
  T.sbuf = static_cast<double2*>(vp);
  if ((rc = alloc(op.get(), sizeof(int) * 4, &vp))) return rc;
  T.err = static_cast<int*>(vp);
  cudaMemset(T.err, 0, sizeof(int) * 4);

  for (int a = 0; a < 3; ++a) {
    const int n = dims[a];
    std::vector<double> tw = twiddles(n);
    if ((rc = upload(op.get(), tw.data(), tw.size(), &d_dbl))) return rc;
    const double2* p2 = reinterpret_cast<const double2*>(d_dbl);
    if (a == 0) G.tw0 = p2;
    if (a == 1) G.tw1 = p2;
    if (a == 2) G.tw2 = p2;
    std::vector<float> twf(tw.size());
    for (size_t i = 0; i < tw.size(); ++i) twf[i] = (float)tw[i];
    float* d_tf;
    if ((rc = upload(op.get(), twf.data(), twf.size(), &d_tf))) return rc;
    const float2* f2 = reinterpret_cast<const float2*>(d_tf);
    if (a == 0) G.tw0f = f2;
    if (a == 1) G.tw1f = f2;
    if (a == 2) G.tw2f = f2;
  }

  // nonlocal operands and the static diagonal
  NlDev& N = op->nl;
  N.rows = (int)npw;
  op->shape.nproj = nproj;
  op->diag.assign(npw, 0.0);
  op->diag = kin;  // no projectors: the diagonal is the kinetic term
  if (nproj > 0) {
    const int natoms = pr->natoms;
    std::vector<int> atom_off{0}, d_off;
    int doff = 0, maxch = 0;
    for (int a = 0; a < natoms; ++a) {
      const int c = pr->channels[a];
      if (c < 1 || c > 64) return fail(ctx, BG_ESHAPE, "channels per atom must be 1..64");
      d_off.push_back(doff);
      doff += c * c;
      atom_off.push_back(atom_off.back() + c);
      maxch = std::max(maxch, c);
    }
    if (atom_off.back() != nproj) return fail(ctx, BG_ESHAPE, "channel counts do not sum to nproj");
    for (int i = 0; i < doff; ++i)
      if (!std::isfinite(pr->couplings[i])) return fail(ctx, BG_ENONFINITE, "coupling not finite");
    const std::complex<double>* P = reinterpret_cast<const std::complex<double>*>(pr->table);
    for (int64_t i = 0; i < npw * nproj; ++i)
      if (!std::isfinite(P[i].real()) || !std::isfinite(P[i].imag()))
        return fail(ctx, BG_ENONFINITE, "projector table not finite");
    // static diagonal (complex: distributed_complex.rs:29-53; Gamma: refstart.rs:605-650)
    std::vector<double> dfull(npw);
    for (int64_t g = 0; g < npw; ++g) dfull[g] = b->kinetic[g];
    // blocks of G on the host threads; each G sums atoms and channel pairs in order
    const int64_t gblk = 2048;
#pragma omp parallel for schedule(dynamic)
    for (int64_t g0 = 0; g0 < npw; g0 += gblk) {
      const int64_t g1 = std::min(npw, g0 + gblk);
      for (int a = 0, off = 0; a < natoms; ++a) {
        const int c = pr->channels[a];
        const double* D = pr->couplings + d_off[a];
        for (int i = 0; i < c; ++i)
          for (int j = 0; j < c; ++j) {
            const double d = D[i * c + j];
            if (d == 0.0) continue;
            const std::complex<double>* pi = P + (size_t)(off + i) * npw;
            const std::complex<double>* pj = P + (size_t)(off + j) * npw;
            for (int64_t g = g0; g < g1; ++g) dfull[g] += (d * pi[g] * std::conj(pj[g])).real();
          }
        off += c;
      }
    }
    if (gamma) {
      op->diag[0] = dfull[0];
      for (size_t i = 1; i < plus.size(); ++i) op->diag[2 * i - 1] = op->diag[2 * i] = dfull[plus[i]];
      // ORC projector rows (distributed_real_gamma.rs:358-398)
      std::vector<double> porc((size_t)npw * nproj);
      const double r2 = std::sqrt(2.0);
      for (int p = 0; p < nproj; ++p) {
        const std::complex<double>* col = P + (size_t)p * npw;
        double* o = porc.data() + (size_t)p * npw;
        o[0] = col[0].real();
        for (size_t i = 1; i < plus.size(); ++i) {
          o[2 * i - 1] = r2 * col[plus[i]].real();
          o[2 * i] = r2 * col[plus[i]].imag();
        }
      }
      if ((rc = upload(op.get(), porc.data(), porc.size(), &d_dbl))) return rc;
    } else {
      op->diag = dfull;
      if ((rc = upload(op.get(), pr->table, (size_t)2 * npw * nproj, &d_dbl))) return rc;
      // P as bf16 hi/lo panels for the tensor-core products of the precision form (split
      // once: the table is constant for the operator's lifetime)
      if ((rc = alloc(op.get(), tc::a_panel_bytes(nproj, npw), &vp))) return rc;
      N.p_tn = static_cast<const unsigned char*>(vp);
      if ((rc = alloc(op.get(), tc::a_panel_bytes((int)npw, nproj), &vp))) return rc;
      N.p_nn = static_cast<const unsigned char*>(vp);
      N.kt_tn = tc::k_tiles(npw);
      N.kt_nn = tc::k_tiles(nproj);
      const double2* pd = reinterpret_cast<const double2*>(d_dbl);
      ce = tc::split_a(tc::kTN, pd, npw, nproj, (int)npw, const_cast<unsigned char*>(N.p_tn), nullptr);
      if (ce == cudaSuccess)
        ce = tc::split_a(tc::kNN, pd, npw, (int)npw, nproj, const_cast<unsigned char*>(N.p_nn), nullptr);
      if (ce != cudaSuccess) return cuda_fail(ctx, ce, "projector panels");
    }
    N.p = d_dbl;
    op->shape.natoms = natoms;
    op->shape.maxch = maxch;
    if ((rc = upload(op.get(), atom_off.data(), atom_off.size(), &d_int))) return rc;
    N.atom_off = d_int;
    if ((rc = upload(op.get(), d_off.data(), d_off.size(), &d_int))) return rc;
    N.d_off = d_int;
    if ((rc = upload(op.get(), pr->couplings, (size_t)doff, &d_dbl))) return rc;
    N.d = d_dbl;
    int64_t maxpart = 0;
    for (int64_t c = 1; c <= capacity; ++c) {
      int kc;
      const int ks = ksplit_for(npw, nproj, c, &kc);
      maxpart = std::max<int64_t>(maxpart, (int64_t)ks * c);
    }
    const size_t es = gamma ? sizeof(double) : sizeof(double2);
    op->part_cols = maxpart;
    if ((rc = alloc(op.get(), es * (size_t)maxpart * nproj, &vp))) return rc;
    N.part = static_cast<double*>(vp);
    if ((rc = alloc(op.get(), es * (size_t)capacity * nproj, &vp))) return rc;
    N.wd = static_cast<double*>(vp);
  }
  for (double v : op->diag)
    if (!std::isfinite(v)) return fail(ctx, BG_ENONFINITE, "nonfinite diagonal");

  const size_t es = gamma ? sizeof(double) : sizeof(double2);
  if ((rc = alloc(op.get(), es * (size_t)npw * capacity, &vp, &op->xs))) return rc;
  if ((rc = alloc(op.get(), es * (size_t)npw * capacity, &vp, &op->ys))) return rc;
  if ((ce = cudaMallocHost(&op->err_host, sizeof(int) * 4)) != cudaSuccess) return cuda_fail(ctx, ce, "cudaMallocHost");
  if ((ce = cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, ce, "cudaStreamCreate");
  op->own_stream = true;
  const size_t ps = plane_smem_bytes(G), ss = stick_smem_bytes(G);
  int dev_smem = 0;
  cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  if (ps > (size_t)dev_smem || ss > (size_t)dev_smem)
    return fail(ctx, BG_ESHAPE, "FFT plane does not fit in shared memory");
  if ((rc = configure_kernels((size_t)dev_smem, (size_t)dev_smem)) != BG_OK)
    return fail(ctx, BG_EDEVICE, "cudaFuncSetAttribute failed");
  if ((rc = upload(op.get(), &op->t, 1, &op->d_tabs))) return rc;
  if ((rc = upload(op.get(), &op->nl, 1, &op->d_nl))) return rc;
  for (int i = 0; i < 2 * kStages; ++i)
    if ((ce = cudaEventCreate(&op->ev.ev[i])) != cudaSuccess) return cuda_fail(ctx, ce, "cudaEventCreate");
  if ((ce = cudaDeviceSynchronize()) != cudaSuccess) return cuda_fail(ctx, ce, "setup");
  *out = op.release();
  return BG_OK;
}

// Wait for the operator stream and report (then clear) the device error word:
// bit 0 a non-finite coefficient read by a kernel, bit 1 a non-finite potential value.
int check_err(bg_op* op) {
  cudaError_t e = cudaMemcpyAsync(op->err_host, op->t.err, sizeof(int), cudaMemcpyDeviceToHost, op->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(op->stream);
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "apply");
  const int bits = op->err_host[0];
  if (bits) {
    cudaMemsetAsync(op->t.err, 0, sizeof(int), op->stream);
    cudaStreamSynchronize(op->stream);
    return fail(op->ctx, BG_ENONFINITE, (bits & 2) ? "non-finite potential value" : "non-finite input coefficient");
  }
  return BG_OK;
}

// Lazily allocated operator buffers (kept for the operator's lifetime).
int ensure_buf(bg_op* op, double** p, size_t doubles) {
  if (*p) return BG_OK;
  void* vp = nullptr;
  int rc = alloc(op, doubles * sizeof(double), &vp);
  if (rc) return rc;
  *p = static_cast<double*>(vp);
  return BG_OK;
}

size_t grid_points(const bg_op* op) { return (size_t)op->dims[0] * op->dims[1] * op->dims[2]; }

// Install a C-order grid (device pointer) into `dst` in the layout of t.vt; waits and
// reports a non-finite value before returning, leaving `dst` unspecified in that case.
int transpose_grid(bg_op* op, const double* v_dev, double* dst) {
  launch_potential_transpose(v_dev, op->g, dst, op->t.err, op->stream);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "kernel launch");
  return check_err(op);
}

// Stage a grid given by pointer kind on the device (host grids go through op->grid).
int grid_on_device(bg_op* op, const double* v, int32_t ptr_kind, const double** out) {
  if (ptr_kind == BG_PTR_DEVICE) {
    *out = v;
    return BG_OK;
  }
  int rc = ensure_buf(op, &op->grid, grid_points(op));
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(op->grid, v, grid_points(op) * sizeof(double), cudaMemcpyHostToDevice, op->stream);
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "copy in");
  *out = op->grid;
  return BG_OK;
}

}  // namespace

extern "C" {

int bg_ctx_create(const bg_device_opts* opts, bg_ctx** out) {
  if (!out) return fail(nullptr, BG_EINVAL, "null output");
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return fail(nullptr, BG_EDEVICE, "no CUDA device available");
  const int dev = opts ? opts->device : 0;
  if (dev < 0 || dev >= count) return fail(nullptr, BG_EINVAL, "device ordinal out of range");
  cudaDeviceProp prop;
  if ((e = cudaGetDeviceProperties(&prop, dev)) != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceProperties");
  if (prop.major != 10) return fail(nullptr, BG_EDEVICE, "libbaandi_b200 is built for sm_100a (B200)");
  auto* c = new bg_ctx();
  c->device = dev;
  *out = c;
  return BG_OK;
}

int bg_ctx_destroy(bg_ctx* ctx) {
  delete ctx;
  return BG_OK;
}

int bg_last_error(const bg_ctx* ctx, char* buf, size_t len) {
  if (!buf || len == 0) return BG_EINVAL;
  const std::string msg = ctx ? ctx->error : global_error();
  std::snprintf(buf, len, "%s", msg.c_str());
  return BG_OK;
}

int bg_op_create_complex(bg_ctx* ctx, const bg_basis_desc* basis, const bg_projectors* proj, int64_t capacity,
                         bg_op** out) {
  return build_op(ctx, basis, proj, capacity, false, out);
}

int bg_op_create_gamma_real(bg_ctx* ctx, const bg_basis_desc* basis, const bg_projectors* proj, int64_t capacity,
                            bg_op** out) {
  return build_op(ctx, basis, proj, capacity, true, out);
}

int bg_op_destroy(bg_op* op) {
  if (!op) return BG_OK;
  if (op->stream) cudaStreamSynchronize(op->stream);
  for (int i = 0; i < 2 * kStages; ++i)
    if (op->ev.ev[i]) cudaEventDestroy(op->ev.ev[i]);
  if (op->own_stream && op->stream) cudaStreamDestroy(op->stream);
  if (op->err_host) cudaFreeHost(op->err_host);
  op->tc.release();
  delete op;
  return BG_OK;
}

int bg_op_set_potential(bg_op* op, const double* v, uint64_t epoch) {
  if (!op || !v) return fail(op ? op->ctx : nullptr, BG_EINVAL, "null argument");
  if (op->has_epoch && epoch <= op->epoch) return fail(op->ctx, BG_EEPOCH, "potential epoch must increase");
  const int n0 = op->dims[0], n1 = op->dims[1], n2 = op->dims[2];
  const size_t vs = (size_t)op->g.vstride;
  std::vector<double> vt(vs * n2, 0.0);
  for (int x = 0; x < n0; ++x)
    for (int y = 0; y < n1; ++y)
      for (int z = 0; z < n2; ++z) {
        const double w = v[((size_t)x * n1 + y) * n2 + z];
        if (!std::isfinite(w)) return fail(op->ctx, BG_ENONFINITE, "potential not finite");
        vt[(size_t)z * vs + (size_t)y * n0 + x] = w;
      }
  cudaError_t e = cudaMemcpyAsync(const_cast<double*>(op->t.vt), vt.data(), vt.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, op->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(op->stream);
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "set_potential");
  op->vtf_valid = false;
  op->epoch = epoch;
  op->has_epoch = true;
  return BG_OK;
}

int bg_op_apply_block(bg_op* op, const double* x, double* y, int64_t rows, int64_t cols, int32_t ptr_kind,
                      int32_t precision) {
  if (!op) return fail(nullptr, BG_EINVAL, "null operator");
  bg_ctx* ctx = op->ctx;
  if (precision != BG_PREC_FP64 && precision != BG_PREC_FP32 && precision != BG_PREC_TENSOR)
    return fail(ctx, BG_EINVAL, "unsupported precision");
  if (precision != BG_PREC_FP64 && (op->is_dense || !fp32_supported(op->g)))
    return fail(ctx, BG_EINVAL, "the FP32 apply needs a cubic grid of 25, 45, 54, 60, 72 or 108 points");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  if (!op->has_epoch) return fail(ctx, BG_EEPOCH, "potential was never set");
  if (rows != op->rows || cols < 0 || cols > op->cap) return fail(ctx, BG_ESHAPE, "block shape");
  if (cols == 0) return BG_OK;
  if (!x || !y || x == y) return fail(ctx, BG_EINVAL, "x and y must be distinct non-null buffers");
  const size_t dpc = op->gamma ? (size_t)rows : (size_t)2 * rows;  // doubles per column
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const double* dx = x;
  double* dy = y;
  if (ptr_kind == BG_PTR_HOST) {
    // Finiteness is checked on the device by the scatter pass (every input value is
    // read there) and reported after the copy back, before this call returns.
    dx = static_cast<const double*>(op->xs->p);
    dy = static_cast<double*>(op->ys->p);
    e = cudaMemcpyAsync(const_cast<double*>(dx), x, dpc * cols * sizeof(double), cudaMemcpyHostToDevice, op->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy in");
  }
  if (precision != BG_PREC_FP64) {
    int rc = ensure_potential_float(op, op->stream);
    if (rc) return rc;
  }
  const bool tensor_nl = precision == BG_PREC_TENSOR && !op->gamma && op->shape.nproj > 0;
  if (tensor_nl && ensure_nonlocal_tc(&op->tc, 1, op->shape.nproj, (int)op->cap, (int)op->rows))
    return fail(ctx, BG_ENOMEM, "tensor-core nonlocal buffers");
  if (op->is_dense) {
    int rc = dense_apply(op, dx, dy, cols);
    if (rc != BG_OK) return rc;
  } else {
  Batch bt;
  bt.nk = 1;
  CallArgs& a = bt.a[0];
  a.x = dx;
  a.y = dy;
  a.ldx = (int64_t)dpc;
  a.ldy = (int64_t)dpc;
  a.cols = (int)cols;
  a.units = op->gamma ? (int)((cols + 1) / 2) : (int)cols;
  op->launches += launch_local(op->d_tabs, op->gamma ? 1 : 0, op->t.ngroups, op->g, bt, op->stream, &op->ev,
                               precision != BG_PREC_FP64 ? 1 : 0);
  if (tensor_nl) {
    op->launches += launch_nonlocal_tc(op->d_nl, op->shape, (int)op->rows, (int)cols, bt, &op->tc, op->stream, &op->ev);
  } else if (op->shape.nproj > 0) {
    NlShape sh = op->shape;
    sh.ksplit = ksplit_for(op->rows, sh.nproj, cols, &sh.kchunk);
    op->launches += launch_nonlocal(op->d_nl, op->gamma ? 1 : 0, sh, (int)op->rows, bt, op->stream, &op->ev);
  }
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  if (ptr_kind == BG_PTR_HOST) {
    e = cudaMemcpyAsync(y, dy, dpc * cols * sizeof(double), cudaMemcpyDeviceToHost, op->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy out");
    return check_err(op);
  }
  return BG_OK;
}

int bg_op_sync(bg_op* op) {
  if (!op) return fail(nullptr, BG_EINVAL, "null operator");
  return check_err(op);
}

int bg_op_diagonal(const bg_op* op, double* out) {
  if (!op || !out) return fail(op ? op->ctx : nullptr, BG_EINVAL, "null argument");
  std::copy(op->diag.begin(), op->diag.end(), out);
  return BG_OK;
}

int bg_op_rows(const bg_op* op, int64_t* rows) {
  if (!op || !rows) return BG_EINVAL;
  *rows = op->rows;
  return BG_OK;
}

int bg_op_capacity(const bg_op* op, int64_t* capacity) {
  if (!op || !capacity) return BG_EINVAL;
  *capacity = op->cap;
  return BG_OK;
}

int bg_op_stream(const bg_op* op, void** stream) {
  if (!op || !stream) return BG_EINVAL;
  *stream = op->stream;
  return BG_OK;
}

int bg_op_set_stream(bg_op* op, void* stream) {
  if (!op) return BG_EINVAL;
  if (op->own_stream && op->stream) {
    cudaStreamSynchronize(op->stream);
    cudaStreamDestroy(op->stream);
  }
  op->own_stream = false;
  op->stream = static_cast<cudaStream_t>(stream);
  return BG_OK;
}

int bg_op_launches(const bg_op* op, int64_t* launches) {
  if (!op || !launches) return BG_EINVAL;
  *launches = op->launches;
  return BG_OK;
}

int bg_op_profile(bg_op* op, int32_t enable) {
  if (!op) return BG_EINVAL;
  op->ev.on = enable != 0;
  return BG_OK;
}

static int stage_times(bg_ctx* ctx, cudaStream_t stream, const StageEvents& ev, double* ms) {
  if (!ms) return fail(ctx, BG_EINVAL, "null output");
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "stage_times");
  for (int s = 0; s < kStages; ++s) {
    float t = 0.0f;
    ms[s] = 0.0;
    if (ev.on && cudaEventQuery(ev.ev[2 * s]) == cudaSuccess && cudaEventQuery(ev.ev[2 * s + 1]) == cudaSuccess &&
        cudaEventElapsedTime(&t, ev.ev[2 * s], ev.ev[2 * s + 1]) == cudaSuccess)
      ms[s] = t;
  }
  cudaGetLastError();
  return BG_OK;
}

int bg_op_stage_times(bg_op* op, double* ms) {
  if (!op) return BG_EINVAL;
  return stage_times(op->ctx, op->stream, op->ev, ms);
}

int bg_op_set_potential_ptr(bg_op* op, const double* v, uint64_t epoch, int32_t ptr_kind) {
  if (!op || !v) return fail(op ? op->ctx : nullptr, BG_EINVAL, "null argument");
  if (ptr_kind == BG_PTR_HOST) return bg_op_set_potential(op, v, epoch);
  if (ptr_kind != BG_PTR_DEVICE) return fail(op->ctx, BG_EINVAL, "pointer kind");
  if (op->is_dense) return fail(op->ctx, BG_EINVAL, "a dense operator has no potential grid");
  if (op->has_epoch && epoch <= op->epoch) return fail(op->ctx, BG_EEPOCH, "potential epoch must increase");
  cudaError_t e = cudaSetDevice(op->ctx->device);
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "cudaSetDevice");
  // Checked in a scratch copy first so that a rejected potential leaves the old one.
  int rc = ensure_buf(op, &op->vchange, (size_t)op->g.vstride * op->dims[2]);
  if (rc) return rc;
  if ((rc = transpose_grid(op, v, op->vchange))) return rc;
  e = cudaMemcpyAsync(const_cast<double*>(op->t.vt), op->vchange, sizeof(double) * op->g.vstride * op->dims[2],
                      cudaMemcpyDeviceToDevice, op->stream);
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "set_potential");
  op->vtf_valid = false;
  op->epoch = epoch;
  op->has_epoch = true;
  return BG_OK;
}

int bg_op_add_local_change(bg_op* op, const double* x, const double* change, double* hx, int64_t rows, int64_t cols,
                           int32_t ptr_kind) {
  if (!op) return fail(nullptr, BG_EINVAL, "null operator");
  bg_ctx* ctx = op->ctx;
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  if (op->is_dense) return fail(ctx, BG_EINVAL, "a dense operator has no potential grid");
  if (rows != op->rows || cols < 0 || cols > op->cap) return fail(ctx, BG_ESHAPE, "block shape");
  if (!x || !hx || !change || (const double*)hx == x) return fail(ctx, BG_EINVAL, "x, change and hx must be distinct non-null buffers");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  int rc = ensure_buf(op, &op->vchange, (size_t)op->g.vstride * op->dims[2]);
  if (rc) return rc;
  const double* dv = nullptr;
  if ((rc = grid_on_device(op, change, ptr_kind, &dv))) return rc;
  if ((rc = transpose_grid(op, dv, op->vchange))) return rc;  // change checked before hx is touched
  if (cols == 0) return BG_OK;
  const size_t dpc = op->gamma ? (size_t)rows : (size_t)2 * rows;
  const double* dx = x;
  double* dhx = hx;
  if (ptr_kind == BG_PTR_HOST) {
    dx = static_cast<const double*>(op->xs->p);
    dhx = static_cast<double*>(op->ys->p);
    e = cudaMemcpyAsync(const_cast<double*>(dx), x, dpc * cols * sizeof(double), cudaMemcpyHostToDevice, op->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dhx, hx, dpc * cols * sizeof(double), cudaMemcpyHostToDevice, op->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy in");
  }
  Batch bt;
  bt.nk = 1;
  CallArgs& a = bt.a[0];
  a.x = dx;
  a.y = dhx;
  a.ldx = a.ldy = (int64_t)dpc;
  a.cols = (int)cols;
  a.units = op->gamma ? (int)((cols + 1) / 2) : (int)cols;
  a.vt = op->vchange;
  a.accumulate = 1;
  op->launches += launch_local(op->d_tabs, op->gamma ? 1 : 0, op->t.ngroups, op->g, bt, op->stream, nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  if (ptr_kind == BG_PTR_HOST) {
    if ((rc = check_err(op))) return rc;  // hx on the host stays untouched on a non-finite input
    e = cudaMemcpyAsync(hx, dhx, dpc * cols * sizeof(double), cudaMemcpyDeviceToHost, op->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(op->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy out");
  }
  return BG_OK;
}

int bg_op_band_density_sum(bg_op* op, const double* x, int64_t rows, int64_t cols, const double* weights,
                           double volume, double* density, int32_t accumulate, int32_t ptr_kind) {
  if (!op) return fail(nullptr, BG_EINVAL, "null operator");
  bg_ctx* ctx = op->ctx;
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  if (op->is_dense) return fail(ctx, BG_EINVAL, "a dense operator has no grid");
  if (rows != op->rows || cols < 0 || cols > op->cap) return fail(ctx, BG_ESHAPE, "block shape");
  if (!density || (cols > 0 && (!x || !weights))) return fail(ctx, BG_EINVAL, "null argument");
  if (!std::isfinite(volume) || volume <= 0.0) return fail(ctx, BG_ESHAPE, "volume must be finite and positive");
  for (int64_t c = 0; c < cols; ++c)
    if (!std::isfinite(weights[c]) || weights[c] < 0.0)
      return fail(ctx, BG_ESHAPE, "band weights must be finite and non-negative");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const size_t pts = grid_points(op);
  int rc;
  double* dd = density;
  if (ptr_kind == BG_PTR_HOST) {
    if ((rc = ensure_buf(op, &op->grid, pts))) return rc;
    dd = op->grid;
    if (accumulate) {
      e = cudaMemcpyAsync(dd, density, pts * sizeof(double), cudaMemcpyHostToDevice, op->stream);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "copy in");
    }
  }
  if (cols == 0) {
    if (!accumulate) {
      e = cudaMemsetAsync(dd, 0, pts * sizeof(double), op->stream);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "memset");
    }
  } else {
    const int units = op->gamma ? (int)((cols + 1) / 2) : (int)cols;
    // Enough (plane, chunk) blocks for two waves of 148 SMs; chunks sum in order.
    const int max_chunks = std::max<int>(1, std::min<int64_t>(op->cap_units, (2 * 148 + op->dims[2] - 1) / op->dims[2]));
    if (!op->dens_part) {
      if ((rc = ensure_buf(op, &op->dens_part, (size_t)max_chunks * pts))) return rc;
      op->dens_chunks = max_chunks;
    }
    if ((rc = ensure_buf(op, &op->dens_w, (size_t)op->cap))) return rc;
    const int want = std::min(units, op->dens_chunks);
    const int per_chunk = (units + want - 1) / want;
    const int chunks = (units + per_chunk - 1) / per_chunk;
    const size_t dpc = op->gamma ? (size_t)rows : (size_t)2 * rows;
    const double* dx = x;
    if (ptr_kind == BG_PTR_HOST) {
      dx = static_cast<const double*>(op->xs->p);
      e = cudaMemcpyAsync(const_cast<double*>(dx), x, dpc * cols * sizeof(double), cudaMemcpyHostToDevice, op->stream);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "copy in");
    }
    e = cudaMemcpyAsync(op->dens_w, weights, cols * sizeof(double), cudaMemcpyHostToDevice, op->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy in");
    Batch bt;
    bt.nk = 1;
    CallArgs& a = bt.a[0];
    a.x = dx;
    a.y = nullptr;
    a.ldx = a.ldy = (int64_t)dpc;
    a.cols = (int)cols;
    a.units = units;
    op->launches += launch_density(op->d_tabs, op->gamma ? 1 : 0, op->t.ngroups, op->g, bt, op->dens_w, 0, per_chunk,
                                   chunks, op->dens_part, op->stream);
    if ((rc = ensure_buf(op, &op->dens_ksum, pts))) return rc;
    launch_density_reduce(op->dens_part, 1, chunks, op->g, volume, accumulate, op->dens_ksum, dd, op->stream);
    op->launches += 2;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  }
  if (ptr_kind == BG_PTR_HOST) {
    if ((rc = check_err(op))) return rc;
    e = cudaMemcpyAsync(density, dd, pts * sizeof(double), cudaMemcpyDeviceToHost, op->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(op->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy out");
  }
  return BG_OK;
}

}  // extern "C"

namespace bg {
// Launch the local and nonlocal stages of operators [k0, k1) of a set on one stream.
int ensure_potential_float(bg_op* op, cudaStream_t s) {
  if (op->vtf_valid || op->is_dense) return BG_OK;
  launch_potential_float(op->t.vt, op->g, const_cast<float*>(op->t.vtf), s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(op->ctx, e, "kernel launch");
  op->vtf_valid = true;
  return BG_OK;
}

int enqueue_range(bg_kset* ks, int k0, int k1, const CallArgs* args, const int64_t* cols, cudaStream_t s,
                  StageEvents* ev, int prec, TcNl* tc) {
  Batch bt;
  bt.nk = k1 - k0;
  int max_groups = 0, max_rows = 0;
  int64_t max_cols = 0;
  for (int k = k0; k < k1; ++k) {
    bt.a[k - k0] = args[k];
    max_groups = std::max(max_groups, ks->ops[k]->t.ngroups);
    max_rows = std::max(max_rows, (int)ks->ops[k]->rows);
    max_cols = std::max(max_cols, cols[k]);
  }
  if (max_cols == 0) return 0;
  int launches = launch_local(ks->d_tabs + k0, ks->gamma, max_groups, ks->g, bt, s, ev, prec != BG_PREC_FP64 ? 1 : 0);
  if (prec == BG_PREC_TENSOR && !ks->gamma && ks->shape.nproj > 0) {
    launches += launch_nonlocal_tc(ks->d_nl + k0, ks->shape, max_rows, (int)max_cols, bt, tc ? tc : &ks->tc, s, ev);
  } else if (ks->shape.nproj > 0) {
    NlShape sh = ks->shape;
    int64_t tiles = 0, cap = 1 << 30;
    for (int k = k0; k < k1; ++k) {
      tiles += ((sh.nproj + 47) / 48) * ((cols[k] + 47) / 48);
      if (cols[k] > 0) cap = std::min<int64_t>(cap, ks->ops[k]->part_cols / cols[k]);
    }
    sh.ksplit = ksplit_tiles(max_rows, std::max<int64_t>(tiles, 1), &sh.kchunk, cap);
    launches += launch_nonlocal(ks->d_nl + k0, ks->gamma, sh, max_rows, bt, s, ev);
  }
  return launches;
}
}  // namespace bg

extern "C" {

int bg_kset_create(bg_ctx* ctx, int32_t n, bg_op* const* ops, bg_kset** out) {
  if (!ctx || !ops || !out) return fail(ctx, BG_EINVAL, "null argument");
  if (n < 1 || n > kMaxBatch) return fail(ctx, BG_ESHAPE, "a k-point set holds 1..64 operators");
  auto ks = std::make_unique<bg_kset>();
  ks->ctx = ctx;
  const bg_op* o0 = ops[0];
  if (!o0) return fail(ctx, BG_EINVAL, "null operator");
  std::vector<OpTables> tabs;
  std::vector<NlDev> nls;
  for (int i = 0; i < n; ++i) {
    const bg_op* o = ops[i];
    if (!o || o->ctx != ctx) return fail(ctx, BG_EINVAL, "operators must belong to this context");
    if (o->is_dense != o0->is_dense) return fail(ctx, BG_EINVAL, "a k-point set is all dense or all grid operators");
    if (o->gamma != o0->gamma || std::memcmp(o->dims, o0->dims, sizeof o->dims) != 0 ||
        o->shape.nproj != o0->shape.nproj || o->shape.natoms != o0->shape.natoms)
      return fail(ctx, BG_ESHAPE, "operators of a set need one grid, one kind and one projector layout");
    ks->ops.push_back(const_cast<bg_op*>(o));
    tabs.push_back(o->t);
    nls.push_back(o->nl);
    ks->max_groups = std::max(ks->max_groups, o->t.ngroups);
    ks->max_rows = std::max<int>(ks->max_rows, (int)o->rows);
    ks->shape.maxch = std::max(ks->shape.maxch, o->shape.maxch);
  }
  ks->gamma = o0->gamma ? 1 : 0;
  ks->dense = o0->is_dense;
  ks->shape.nproj = o0->shape.nproj;
  ks->shape.natoms = o0->shape.natoms;
  ks->g = o0->g;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaMalloc(&ks->d_tabs, sizeof(OpTables) * n);
  if (e == cudaSuccess) e = cudaMalloc(&ks->d_nl, sizeof(NlDev) * n);
  if (e == cudaSuccess) e = cudaMemcpy(ks->d_tabs, tabs.data(), sizeof(OpTables) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ks->d_nl, nls.data(), sizeof(NlDev) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ks->stream, cudaStreamNonBlocking);
  for (int i = 0; i < 2 * kStages && e == cudaSuccess; ++i) e = cudaEventCreate(&ks->ev.ev[i]);
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaStreamCreateWithFlags(&ks->pipe[i], cudaStreamNonBlocking);
  for (int i = 0; i < bg_kset::kChunks && e == cudaSuccess; ++i) {
    e = cudaEventCreateWithFlags(&ks->in_done[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ks->work_done[i], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    if (ks->d_tabs) cudaFree(ks->d_tabs);
    if (ks->d_nl) cudaFree(ks->d_nl);
    return cuda_fail(ctx, e, "k-point set");
  }
  ks->own_stream = true;
  *out = ks.release();
  return BG_OK;
}

int bg_kset_destroy(bg_kset* ks) {
  if (!ks) return BG_OK;
  if (ks->stream) cudaStreamSynchronize(ks->stream);
  for (int i = 0; i < 2 * kStages; ++i)
    if (ks->ev.ev[i]) cudaEventDestroy(ks->ev.ev[i]);
  if (ks->own_stream && ks->stream) cudaStreamDestroy(ks->stream);
  for (int i = 0; i < 3; ++i)
    if (ks->pipe[i]) {
      cudaStreamSynchronize(ks->pipe[i]);
      cudaStreamDestroy(ks->pipe[i]);
    }
  for (int i = 0; i < bg_kset::kChunks; ++i) {
    if (ks->in_done[i]) cudaEventDestroy(ks->in_done[i]);
    if (ks->work_done[i]) cudaEventDestroy(ks->work_done[i]);
  }
  for (int i = 0; i < 2; ++i) {
    if (ks->stage_in[i]) cudaFreeHost(ks->stage_in[i]);
    if (ks->stage_out[i]) cudaFreeHost(ks->stage_out[i]);
    if (ks->in_copied[i]) cudaEventDestroy(ks->in_copied[i]);
    if (ks->out_copied[i]) cudaEventDestroy(ks->out_copied[i]);
  }
  if (ks->dv_cache && ks->dv_free) ks->dv_free(ks->dv_cache);
  cudaFree(ks->d_vts);
  cudaFree(ks->d_errs);
  cudaFree(ks->d_errv);
  if (ks->h_errv) cudaFreeHost(ks->h_errv);
  cudaFree(ks->dens_part);
  cudaFree(ks->dens_ksum);
  cudaFree(ks->dens_w);
  cudaFree(ks->d_tabs);
  cudaFree(ks->d_nl);
  ks->tc.release();
  delete ks;
  return BG_OK;
}

int bg_kset_set_potential_ptr(bg_kset* ks, const double* v, uint64_t epoch, int32_t ptr_kind) {
  if (!ks || !v) return fail(ks ? ks->ctx : nullptr, BG_EINVAL, "null argument");
  bg_ctx* ctx = ks->ctx;
  if (ks->dense) return fail(ctx, BG_EINVAL, "a dense operator has no potential grid");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  const int n = (int)ks->ops.size();
  for (int k = 0; k < n; ++k) {
    const bg_op* op = ks->ops[k];
    if (op->has_epoch && epoch <= op->epoch) return fail(ctx, BG_EEPOCH, "potential epoch must increase");
  }
  if (ptr_kind == BG_PTR_HOST) {
    for (int k = 0; k < n; ++k)
      if (int rc = bg_op_set_potential(ks->ops[k], v, epoch)) return rc;
    return BG_OK;
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  bg_op* op0 = ks->ops[0];
  const size_t vdoubles = (size_t)ks->g.vstride * ks->g.n2;
  int rc = ensure_buf(op0, &op0->vchange, vdoubles);
  if (rc) return rc;
  if (!ks->d_vts) {
    std::vector<double*> h(n);
    for (int k = 0; k < n; ++k) h[k] = const_cast<double*>(ks->ops[k]->t.vt);
    void* p = nullptr;
    if ((e = cudaMalloc(&p, n * sizeof(double*))) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    ks->d_vts = static_cast<double**>(p);
    if ((e = cudaMemcpy(ks->d_vts, h.data(), n * sizeof(double*), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(ctx, e, "cudaMemcpy");
  }
  // transposed and checked once in a scratch copy (a rejected potential leaves the old
  // one everywhere), then copied to every operator
  launch_potential_transpose(v, ks->g, op0->vchange, op0->t.err, ks->stream);
  e = cudaMemcpyAsync(op0->err_host, op0->t.err, sizeof(int), cudaMemcpyDeviceToHost, ks->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ks->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "set_potential");
  if (op0->err_host[0]) {
    cudaMemsetAsync(op0->t.err, 0, sizeof(int), ks->stream);
    cudaStreamSynchronize(ks->stream);
    return fail(ctx, BG_ENONFINITE, "non-finite potential value");
  }
  launch_broadcast(op0->vchange, (int64_t)vdoubles, ks->d_vts, n, ks->stream);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  ks->launches += 2;
  for (int k = 0; k < n; ++k) {
    bg_op* op = ks->ops[k];
    op->vtf_valid = false;
    op->epoch = epoch;
    op->has_epoch = true;
  }
  return BG_OK;
}

int bg_kset_band_density_sum(bg_kset* ks, const double* const* x, int64_t cols, const double* weights, double volume,
                             double* density, int32_t accumulate, int32_t ptr_kind) {
  if (!ks || !density) return fail(ks ? ks->ctx : nullptr, BG_EINVAL, "null argument");
  bg_ctx* ctx = ks->ctx;
  if (ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "the set's band density takes device blocks and grid");
  if (ks->dense) return fail(ctx, BG_EINVAL, "a dense operator has no grid");
  const int n = (int)ks->ops.size();
  for (int k = 0; k < n; ++k)
    if (cols < 0 || cols > ks->ops[k]->cap) return fail(ctx, BG_ESHAPE, "block shape");
  if (cols > 0 && (!x || !weights)) return fail(ctx, BG_EINVAL, "null argument");
  for (int k = 0; cols > 0 && k < n; ++k)
    if (!x[k]) return fail(ctx, BG_EINVAL, "null block");
  if (!std::isfinite(volume) || volume <= 0.0) return fail(ctx, BG_ESHAPE, "volume must be finite and positive");
  for (int64_t i = 0; i < cols * n; ++i)
    if (!std::isfinite(weights[i]) || weights[i] < 0.0)
      return fail(ctx, BG_ESHAPE, "band weights must be finite and non-negative");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const BoxGeo& g = ks->g;
  const size_t pts = (size_t)g.n0 * g.n1 * g.n2;
  if (cols == 0) {
    if (!accumulate && (e = cudaMemsetAsync(density, 0, pts * sizeof(double), ks->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "memset");
    return BG_OK;
  }
  const int units = ks->gamma ? (int)((cols + 1) / 2) : (int)cols;
  // one unit per (plane, chunk, k) block while the partial slices fit in 1 GiB (the plane
  // kernel then carries nothing across units and runs four blocks per SM); otherwise
  // enough blocks for two waves of 148 SMs.  Chunks sum in order.
  const bool one = (double)n * units * pts * sizeof(double) <= 1073741824.0;
  const int want = one ? units : std::max(1, std::min(units, (2 * 148 + g.n2 * n - 1) / (g.n2 * n)));
  const int per_chunk = (units + want - 1) / want;
  const int chunks = (units + per_chunk - 1) / per_chunk;
  auto grow = [&](double** p, size_t* have, size_t need) -> int {
    if (*have >= need) return BG_OK;
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
    void* q = nullptr;
    cudaError_t ee = cudaMalloc(&q, need * sizeof(double));
    if (ee != cudaSuccess) return cuda_fail(ctx, ee, "cudaMalloc");
    *p = static_cast<double*>(q);
    *have = need;
    return BG_OK;
  };
  int rc;
  if ((rc = grow(&ks->dens_part, &ks->dens_part_doubles, (size_t)n * chunks * pts))) return rc;
  if ((rc = grow(&ks->dens_w, &ks->dens_w_doubles, (size_t)n * cols))) return rc;
  if ((rc = grow(&ks->dens_ksum, &ks->dens_ksum_doubles, (size_t)n * pts))) return rc;
  e = cudaMemcpyAsync(ks->dens_w, weights, (size_t)n * cols * sizeof(double), cudaMemcpyHostToDevice, ks->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "copy in");
  Batch bt;
  bt.nk = n;
  for (int k = 0; k < n; ++k) {
    const bg_op* op = ks->ops[k];
    const int64_t dpc = op->gamma ? op->rows : 2 * op->rows;
    CallArgs& a = bt.a[k];
    a.x = x[k];
    a.y = nullptr;
    a.ldx = a.ldy = dpc;
    a.cols = (int)cols;
    a.units = units;
  }
  ks->launches += launch_density(ks->d_tabs, ks->gamma, ks->max_groups, g, bt, ks->dens_w, (int)cols, per_chunk,
                                 chunks, ks->dens_part, ks->stream);
  launch_density_reduce(ks->dens_part, n, chunks, g, volume, accumulate, ks->dens_ksum, density, ks->stream);
  ks->launches += 2;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  return BG_OK;
}

int bg_kset_apply(bg_kset* ks, const double* const* x, double* const* y, const int64_t* cols, int32_t ptr_kind,
                  int32_t precision) {
  if (!ks || !x || !y || !cols) return fail(ks ? ks->ctx : nullptr, BG_EINVAL, "null argument");
  bg_ctx* ctx = ks->ctx;
  if (precision != BG_PREC_FP64 && precision != BG_PREC_FP32 && precision != BG_PREC_TENSOR)
    return fail(ctx, BG_EINVAL, "unsupported precision");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  if (ks->dense) return fail(ctx, BG_EINVAL, "a set of dense operators only runs bg_kset_davidson_solve");
  if (precision != BG_PREC_FP64 && !fp32_supported(ks->g))
    return fail(ctx, BG_EINVAL, "the FP32 apply needs a cubic grid of 25, 45, 54, 60, 72 or 108 points");
  const int fp32 = precision != BG_PREC_FP64 ? 1 : 0;
  const int n = (int)ks->ops.size();
  Batch bt;
  bt.nk = n;
  int64_t max_cols = 0;
  for (int k = 0; k < n; ++k) {
    bg_op* op = ks->ops[k];
    if (!op->has_epoch) return fail(ctx, BG_EEPOCH, "potential was never set on an operator of the set");
    if (cols[k] < 0 || cols[k] > op->cap) return fail(ctx, BG_ESHAPE, "block shape");
    if (cols[k] > 0 && (!x[k] || !y[k] || x[k] == y[k]))
      return fail(ctx, BG_EINVAL, "x and y must be distinct non-null buffers");
    max_cols = std::max(max_cols, cols[k]);
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  if (fp32) {
    bool converted = false;
    for (int k = 0; k < n; ++k) {
      converted = converted || !ks->ops[k]->vtf_valid;
      if (int rc = ensure_potential_float(ks->ops[k], ks->stream)) return rc;
    }
    // the host-buffer path runs on its own streams
    if (converted && ptr_kind == BG_PTR_HOST && (e = cudaStreamSynchronize(ks->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "FP32 potential");
  }
  std::vector<CallArgs> args(n);
  for (int k = 0; k < n; ++k) {
    bg_op* op = ks->ops[k];
    const size_t dpc = op->gamma ? (size_t)op->rows : (size_t)2 * op->rows;
    CallArgs& a = args[k];
    a.x = x[k];
    a.y = y[k];
    if (ptr_kind == BG_PTR_HOST) {
      a.x = static_cast<const double*>(op->xs->p);
      a.y = static_cast<double*>(op->ys->p);
    }
    a.ldx = a.ldy = (int64_t)dpc;
    a.cols = (int)cols[k];
    a.units = op->gamma ? (int)((cols[k] + 1) / 2) : (int)cols[k];
  }
  if (max_cols == 0) return BG_OK;
  if (precision == BG_PREC_TENSOR && !ks->gamma && ks->shape.nproj > 0 &&
      ensure_nonlocal_tc(&ks->tc, n, ks->shape.nproj, (int)max_cols, ks->max_rows))
    return fail(ctx, BG_ENOMEM, "tensor-core nonlocal buffers");
  if (ptr_kind == BG_PTR_DEVICE) {
    ks->launches += enqueue_range(ks, 0, n, args.data(), cols, ks->stream, &ks->ev, precision);
    e = cudaGetLastError();
    return e == cudaSuccess ? BG_OK : cuda_fail(ctx, e, "kernel launch");
  }
  // Host buffers: chunks (whole operators of one set, up to kChunkBytes together, or
  // column blocks of one operator larger than that) flow through copy-in, compute and
  // copy-out streams, so the transfers of one chunk overlap the kernels of its neighbours.
  // Pageable blocks go through pinned staging slots that host threads fill and drain while
  // the GPU works on the neighbouring chunks; pinned blocks are copied directly.
  struct Unit {
    int k;
    int64_t c0, c1;  // columns
  };
  struct Chunk {
    int k0, k1;  // operators [k0, k1); a column block when k1 == k0 + 1 and the unit is partial
    std::vector<Unit> units;
    size_t bytes = 0;
  };
  auto dpc_of = [&](int k) { return ks->ops[k]->gamma ? (size_t)ks->ops[k]->rows : (size_t)2 * ks->ops[k]->rows; };
  size_t total = 0;
  for (int k = 0; k < n; ++k) total += dpc_of(k) * sizeof(double) * (size_t)cols[k];
  const size_t kChunkBytes = std::min(kChunkMax, std::max(kChunkMin, total / 8));
  std::vector<Chunk> chunks;
  for (int k = 0; k < n; ++k) {
    if (cols[k] == 0) continue;
    const size_t bpc = dpc_of(k) * sizeof(double);
    const size_t bytes = bpc * (size_t)cols[k];
    if (bytes > kChunkBytes) {
      // column blocks of about kChunkBytes (even starts, so Gamma column pairs stay whole)
      int64_t nb = (int64_t)((bytes + kChunkBytes - 1) / kChunkBytes);
      int64_t per = (cols[k] + nb - 1) / nb;
      per += per & 1;
      for (int64_t c0 = 0; c0 < cols[k]; c0 += per) {
        Chunk ch;
        ch.k0 = k;
        ch.k1 = k + 1;
        ch.units.push_back({k, c0, std::min(cols[k], c0 + per)});
        ch.bytes = bpc * (size_t)(ch.units[0].c1 - c0);
        chunks.push_back(ch);
      }
      continue;
    }
    if (chunks.empty() || chunks.back().k1 != k || chunks.back().bytes + bytes > kChunkBytes ||
        chunks.back().units.back().c1 != cols[chunks.back().units.back().k]) {
      Chunk ch;
      ch.k0 = k;
      ch.k1 = k;
      chunks.push_back(ch);
    }
    chunks.back().units.push_back({k, 0, cols[k]});
    chunks.back().k1 = k + 1;
    chunks.back().bytes += bytes;
  }
  // which side of each operator is pageable (staged) and the staging slots
  std::vector<char> x_staged(n, 0), y_staged(n, 0);
  size_t slot = 0;
  for (int k = 0; k < n; ++k) {
    if (cols[k] == 0) continue;
    x_staged[k] = host_is_pageable(x[k]);
    y_staged[k] = host_is_pageable(y[k]);
  }
  for (const Chunk& ch : chunks) slot = std::max(slot, ch.bytes);
  bool any_staged = false;
  for (int k = 0; k < n; ++k) any_staged = any_staged || x_staged[k] || y_staged[k];
  if (any_staged && slot > ks->stage_bytes) {
    for (int i = 0; i < 2; ++i) {
      if (ks->stage_in[i]) cudaFreeHost(ks->stage_in[i]);
      if (ks->stage_out[i]) cudaFreeHost(ks->stage_out[i]);
      ks->stage_in[i] = ks->stage_out[i] = nullptr;
    }
    ks->stage_bytes = 0;
    for (int i = 0; i < 2; ++i) {
      if ((e = cudaMallocHost(&ks->stage_in[i], slot)) != cudaSuccess ||
          (e = cudaMallocHost(&ks->stage_out[i], slot)) != cudaSuccess)
        return cuda_fail(ctx, e, "pinned staging");
      if (!ks->in_copied[i] && (e = cudaEventCreateWithFlags(&ks->in_copied[i], cudaEventDisableTiming)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaEventCreate");
      if (!ks->out_copied[i] && (e = cudaEventCreateWithFlags(&ks->out_copied[i], cudaEventDisableTiming)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaEventCreate");
    }
    ks->stage_bytes = slot;
  }
  cudaStream_t in = ks->pipe[0], work = ks->pipe[1], out = ks->pipe[2];
  int rc_drain = BG_OK;
  std::vector<CallArgs> cargs(args);
  std::vector<int64_t> ccols(cols, cols + n);
  // the pageable outputs of chunk i wait in out slot i % 2 until the host copies them out
  auto drain = [&](int i) -> int {
    const Chunk& ch = chunks[i];
    bool staged = false;
    for (const Unit& u : ch.units) staged = staged || y_staged[u.k];
    if (!staged) return BG_OK;
    cudaError_t ee = cudaEventSynchronize(ks->out_copied[i % 2]);
    if (ee != cudaSuccess) return cuda_fail(ctx, ee, "copy out");
    size_t off = 0;
    for (const Unit& u : ch.units) {
      const size_t b = dpc_of(u.k) * sizeof(double) * (size_t)(u.c1 - u.c0);
      if (y_staged[u.k])
        parallel_copy(reinterpret_cast<char*>(y[u.k]) + dpc_of(u.k) * sizeof(double) * (size_t)u.c0,
                      static_cast<const char*>(ks->stage_out[i % 2]) + off, b);
      off += b;
    }
    return BG_OK;
  };
  for (int i = 0; i < (int)chunks.size(); ++i) {
    const Chunk& ch = chunks[i];
    const int sl = i % 2;
    // copy in: pageable units packed into in slot sl once chunk i - 2 has left it
    bool xst = false;
    for (const Unit& u : ch.units) xst = xst || x_staged[u.k];
    if (xst && i >= 2 && (e = cudaEventSynchronize(ks->in_copied[sl])) != cudaSuccess)
      return cuda_fail(ctx, e, "copy in");
    size_t off = 0;
    for (const Unit& u : ch.units) {
      const size_t dpc = dpc_of(u.k), b = dpc * sizeof(double) * (size_t)(u.c1 - u.c0);
      const char* src = reinterpret_cast<const char*>(x[u.k]) + dpc * sizeof(double) * (size_t)u.c0;
      char* dst = reinterpret_cast<char*>(const_cast<double*>(args[u.k].x)) + dpc * sizeof(double) * (size_t)u.c0;
      if (x_staged[u.k]) {
        char* st = static_cast<char*>(ks->stage_in[sl]) + off;
        parallel_copy(st, src, b);
        src = st;
      }
      if ((e = cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, in)) != cudaSuccess)
        return cuda_fail(ctx, e, "copy in");
      off += b;
    }
    if (xst) cudaEventRecord(ks->in_copied[sl], in);
    cudaEventRecord(ks->in_done[i % bg_kset::kChunks], in);
    cudaStreamWaitEvent(work, ks->in_done[i % bg_kset::kChunks], 0);
    // compute: whole operators, or the chunk's column block of one operator
    for (const Unit& u : ch.units) {
      const size_t dpc = dpc_of(u.k);
      CallArgs& a = cargs[u.k];
      a = args[u.k];
      a.x = args[u.k].x + dpc * (size_t)u.c0;
      a.y = args[u.k].y + dpc * (size_t)u.c0;
      a.cols = (int)(u.c1 - u.c0);
      a.units = ks->ops[u.k]->gamma ? (int)((a.cols + 1) / 2) : a.cols;
      ccols[u.k] = u.c1 - u.c0;
    }
    ks->launches += enqueue_range(ks, ch.k0, ch.k1, cargs.data(), ccols.data(), work, nullptr, precision);
    cudaEventRecord(ks->work_done[i % bg_kset::kChunks], work);
    cudaStreamWaitEvent(out, ks->work_done[i % bg_kset::kChunks], 0);
    // copy out: chunk i - 2's staged outputs leave out slot sl first
    if (i >= 2 && (rc_drain = drain(i - 2)) != BG_OK) return rc_drain;
    bool yst = false;
    off = 0;
    for (const Unit& u : ch.units) {
      const size_t dpc = dpc_of(u.k), b = dpc * sizeof(double) * (size_t)(u.c1 - u.c0);
      const char* src = reinterpret_cast<const char*>(args[u.k].y) + dpc * sizeof(double) * (size_t)u.c0;
      char* dst = y_staged[u.k] ? static_cast<char*>(ks->stage_out[sl]) + off
                                : reinterpret_cast<char*>(y[u.k]) + dpc * sizeof(double) * (size_t)u.c0;
      yst = yst || y_staged[u.k];
      if ((e = cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, out)) != cudaSuccess)
        return cuda_fail(ctx, e, "copy out");
      off += b;
    }
    if (yst) cudaEventRecord(ks->out_copied[sl], out);
  }
  for (int i = std::max(0, (int)chunks.size() - 2); i < (int)chunks.size(); ++i)
    if ((rc_drain = drain(i)) != BG_OK) return rc_drain;
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  for (int i = 0; i < 3; ++i) {
    e = cudaStreamSynchronize(ks->pipe[i]);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "k-point set");
  }
  return bg_kset_sync(ks);
}

int bg_kset_sync(bg_kset* ks) {
  if (!ks) return BG_EINVAL;
  const int n = (int)ks->ops.size();
  cudaError_t e = cudaSetDevice(ks->ctx->device);
  if (e != cudaSuccess) return cuda_fail(ks->ctx, e, "cudaSetDevice");
  if (!ks->d_errs) {  // every operator's error word, read and cleared by one small kernel
    std::vector<int*> h(n);
    for (int k = 0; k < n; ++k) h[k] = ks->ops[k]->t.err;
    void* p = nullptr;
    if ((e = cudaMalloc(&p, n * sizeof(int*))) != cudaSuccess) return cuda_fail(ks->ctx, e, "cudaMalloc");
    ks->d_errs = static_cast<int**>(p);
    if ((e = cudaMalloc(&p, n * sizeof(int))) != cudaSuccess) return cuda_fail(ks->ctx, e, "cudaMalloc");
    ks->d_errv = static_cast<int*>(p);
    if ((e = cudaMallocHost(&p, n * sizeof(int))) != cudaSuccess) return cuda_fail(ks->ctx, e, "cudaMallocHost");
    ks->h_errv = static_cast<int*>(p);
    if ((e = cudaMemcpy(ks->d_errs, h.data(), n * sizeof(int*), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(ks->ctx, e, "cudaMemcpy");
  }
  launch_gather_errors(ks->d_errs, n, ks->d_errv, ks->stream);
  e = cudaMemcpyAsync(ks->h_errv, ks->d_errv, n * sizeof(int), cudaMemcpyDeviceToHost, ks->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ks->stream);
  if (e != cudaSuccess) return cuda_fail(ks->ctx, e, "k-point set");
  for (int k = 0; k < n; ++k)
    if (ks->h_errv[k]) return fail(ks->ctx, BG_ENONFINITE, "non-finite input coefficient");
  return BG_OK;
}

int bg_kset_stream(const bg_kset* ks, void** stream) {
  if (!ks || !stream) return BG_EINVAL;
  *stream = ks->stream;
  return BG_OK;
}

int bg_kset_set_stream(bg_kset* ks, void* stream) {
  if (!ks) return BG_EINVAL;
  if (ks->own_stream && ks->stream) {
    cudaStreamSynchronize(ks->stream);
    cudaStreamDestroy(ks->stream);
  }
  ks->own_stream = false;
  ks->stream = static_cast<cudaStream_t>(stream);
  return BG_OK;
}

int bg_kset_launches(const bg_kset* ks, int64_t* launches) {
  if (!ks || !launches) return BG_EINVAL;
  *launches = ks->launches;
  return BG_OK;
}

int bg_kset_profile(bg_kset* ks, int32_t enable) {
  if (!ks) return BG_EINVAL;
  ks->ev.on = enable != 0;
  return BG_OK;
}

int bg_kset_stage_times(bg_kset* ks, double* ms) {
  if (!ks) return BG_EINVAL;
  return stage_times(ks->ctx, ks->stream, ks->ev, ms);
}

// ------------------------------------------------------------------ setup ABI
int bg_setup_volume(const double rows[9], double* volume) {
  if (!rows || !volume) return fail(nullptr, BG_EINVAL, "null argument");
  Cell c;
  int rc = cell_init(rows, &c);
  if (rc) return fail(nullptr, rc, "singular or non-finite lattice");
  *volume = c.volume;
  return BG_OK;
}

int bg_setup_basis(const double rows[9], double ecut, const double kfrac[3], int64_t capacity, int64_t* npw,
                   int32_t* miller, double* kpg, double* kpg2) {
  if (!rows || !kfrac || !npw) return fail(nullptr, BG_EINVAL, "null argument");
  Cell c;
  int rc = cell_init(rows, &c);
  if (rc) return fail(nullptr, rc, "singular or non-finite lattice");
  Basis b;
  if ((rc = basis_build(c, ecut, kfrac, &b))) return fail(nullptr, rc, "invalid cutoff");
  *npw = b.npw;
  if (capacity == 0) return BG_OK;
  if (capacity < b.npw || !miller || !kpg || !kpg2) return fail(nullptr, BG_ESHAPE, "output capacity too small");
  std::copy(b.miller.begin(), b.miller.end(), miller);
  std::copy(b.kpg.begin(), b.kpg.end(), kpg);
  std::copy(b.kpg2.begin(), b.kpg2.end(), kpg2);
  return BG_OK;
}

int bg_setup_grid(const double rows[9], double ecut, int32_t dims[3], int32_t required[3]) {
  if (!rows || !dims || !required) return fail(nullptr, BG_EINVAL, "null argument");
  Cell c;
  int rc = cell_init(rows, &c);
  if (rc) return fail(nullptr, rc, "singular or non-finite lattice");
  int d[3], r[3];
  if ((rc = grid_dims(c, ecut, d, r))) return fail(nullptr, rc, "invalid cutoff");
  for (int i = 0; i < 3; ++i) {
    dims[i] = d[i];
    required[i] = r[i];
  }
  return BG_OK;
}

int bg_setup_half_sphere(const int32_t* miller, int64_t npw, int64_t* plus, int64_t* minus) {
  if (!miller || !plus || !minus) return fail(nullptr, BG_EINVAL, "null argument");
  std::vector<int64_t> p, m;
  if (half_sphere(miller, npw, &p, &m)) return fail(nullptr, BG_ESHAPE, "not an inversion-symmetric Gamma sphere");
  std::copy(p.begin(), p.end(), plus);
  std::copy(m.begin(), m.end(), minus);
  return BG_OK;
}

static std::vector<Species> to_species(int32_t n, const bg_species* s) {
  std::vector<Species> out(n);
  for (int i = 0; i < n; ++i)
    out[i] = Species{s[i].z_valence, s[i].mesh,  s[i].r,    s[i].rab, s[i].local,  s[i].nbeta,
                     s[i].l,         s[i].beta_len, s[i].beta, s[i].dij, s[i].natoms, s[i].positions};
  return out;
}

int bg_setup_projector_count(int32_t nspecies, const bg_species* species, int32_t* nproj, int32_t* natoms) {
  if (nspecies < 0 || (nspecies > 0 && !species) || !nproj || !natoms) return fail(nullptr, BG_EINVAL, "argument");
  auto sp = to_species(nspecies, species);
  int np, na;
  int rc = projector_count(nspecies, sp.data(), &np, &na);
  if (rc) return fail(nullptr, rc, "projector angular momentum must be 0..3");
  *nproj = np;
  *natoms = na;
  return BG_OK;
}

int bg_setup_projectors(double volume, int64_t npw, const double* kpg, const double* kpg2, int32_t nspecies,
                        const bg_species* species, double* table, int32_t* channels, double* couplings) {
  if (!kpg || !kpg2 || (nspecies > 0 && !species) || !table || !channels || !couplings)
    return fail(nullptr, BG_EINVAL, "null argument");
  auto sp = to_species(nspecies, species);
  for (auto& s : sp)
    for (int i = 0; i < s.nbeta; ++i)
      if (s.ulen[i] < 1 || s.ulen[i] > s.mesh) return fail(nullptr, BG_ESHAPE, "projector samples exceed the mesh");
  int rc = projectors_build(volume, npw, kpg, kpg2, nspecies, sp.data(),
                            reinterpret_cast<std::complex<double>*>(table), channels, couplings);
  if (rc) return fail(nullptr, rc, "projector table");
  return BG_OK;
}

int bg_setup_ewald(const double rows[9], int32_t natoms, const double* positions, const double* charges,
                   double* energy) {
  if (!rows || !positions || !charges || !energy || natoms < 1) return fail(nullptr, BG_EINVAL, "argument");
  Cell c;
  if (cell_init(rows, &c) != BG_OK) return fail(nullptr, BG_EINVAL, "lattice rows are singular or not finite");
  for (int i = 0; i < 3 * natoms; ++i)
    if (!std::isfinite(positions[i])) return fail(nullptr, BG_ENONFINITE, "ion position not finite");
  const int rc = ewald_energy(c, natoms, positions, charges, energy);
  if (rc) return fail(nullptr, rc, "Ewald energy");
  return BG_OK;
}

int bg_setup_local_form_factor(const bg_species* species, double volume, int64_t n, const double* g, double* out) {
  if (!species || !g || !out || !(volume > 0.0)) return fail(nullptr, BG_EINVAL, "argument");
  auto sp = to_species(1, species);
  int rc = local_form_factor(sp[0], volume, n, g, out);
  if (rc) return fail(nullptr, rc, "local form factor");
  return BG_OK;
}

int bg_setup_atomic_charge(int64_t mesh, const double* r, const double* rab, const double* rho_atom, double volume,
                           int64_t n, const double* q, double* out) {
  if (!r || !rab || !rho_atom || (n > 0 && (!q || !out)) || n < 0 || mesh < 2 || mesh > (1 << 20) ||
      !(volume > 0.0))
    return fail(nullptr, BG_EINVAL, "argument");
  for (int64_t k = 0; k < n; ++k)
    if (!std::isfinite(q[k]) || q[k] < 0.0) return fail(nullptr, BG_EINVAL, "wave number");
  int rc = atomic_charge_transform((int)mesh, r, rab, rho_atom, volume, n, q, out);
  if (rc) return fail(nullptr, rc, "atomic charge transform");
  return BG_OK;
}

}  // extern "C"
