// Operator and context objects shared by the C ABI implementation files.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "bg_internal.h"
#include "hpsi.h"

struct bg_ctx {
  int device = 0;
  std::string error;
  std::mutex mu;
  void* learned = nullptr;  // BF16 parameters of the learned preconditioner (device), or null
  ~bg_ctx() {
    if (learned) cudaFree(learned);
  }
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

struct bg_op {
  bg_ctx* ctx = nullptr;
  bool gamma = false;
  int64_t rows = 0;
  int64_t cap = 0;
  int64_t cap_units = 0;
  int dims[3] = {0, 0, 0};
  bool has_epoch = false;
  uint64_t epoch = 0;
  int64_t launches = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<double> diag;
  bg::OpTables t{};
  bg::BoxGeo g{};
  bg::NlDev nl{};
  bg::NlShape shape{};
  int64_t part_cols = 0;        // capacity of nl.part in (ksplit x columns) units
  bg::OpTables* d_tabs = nullptr;   // device copy of t (a batch of one)
  bg::NlDev* d_nl = nullptr;        // device copy of nl
  bg::StageEvents ev;
  std::vector<std::unique_ptr<DevBuf>> bufs;
  DevBuf* xs = nullptr;  // host-apply staging
  DevBuf* ys = nullptr;
  int* err_host = nullptr;  // pinned
  // Dense operator (tests and fixtures): H is rows x rows on the device.
  bool is_dense = false;
  double* dense = nullptr;
  // Lazily allocated: a potential change in the layout of t.vt, a C-order grid for
  // host potentials and densities, band weights, per-chunk density partial sums.
  double* vchange = nullptr;
  double* grid = nullptr;
  double* dens_w = nullptr;
  double* dens_part = nullptr;
  double* dens_ksum = nullptr;  // one grid: the reduction's per-k sum
  int dens_chunks = 0;  // chunks dens_part holds
  bool vtf_valid = false;  // t.vtf (the FP32 apply's potential) matches t.vt
  bg::TcNl tc;             // tensor-core nonlocal products (BG_PREC_TENSOR)
  // device work arrays of bg_davidson_solve, kept between solves on this operator (the
  // solver takes them in a fixed order and enlarges one only when a solve needs more)
  std::vector<std::unique_ptr<DevBuf>> dv_arena;
};


// A set of operators of one grid applied in batched launches (bg_kset_*).
struct bg_kset {
  bg_ctx* ctx = nullptr;
  std::vector<bg_op*> ops;
  int gamma = 0;
  bool dense = false;  // dense test operators: only bg_kset_davidson_solve accepts the set
  int max_groups = 0;
  int max_rows = 0;
  bg::NlShape shape{};
  bg::BoxGeo g{};
  bg::OpTables* d_tabs = nullptr;
  bg::NlDev* d_nl = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bg::StageEvents ev;
  int64_t launches = 0;
  // host-buffer applies: copy-in, compute and copy-out streams pipelined over chunks
  // (whole operators, or column blocks of one), events reused cyclically
  static constexpr int kChunks = 12;
  cudaStream_t pipe[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t in_done[kChunks] = {}, work_done[kChunks] = {};
  // pageable host blocks: two pinned input and two pinned output staging slots, filled
  // and drained by host threads, and the events that free them
  void* stage_in[2] = {nullptr, nullptr};
  void* stage_out[2] = {nullptr, nullptr};
  size_t stage_bytes = 0;
  cudaEvent_t in_copied[2] = {}, out_copied[2] = {};
  // bg_kset_davidson_solve's solver (work arrays and iteration graph), kept between solves
  void* dv_cache = nullptr;
  void (*dv_free)(void*) = nullptr;
  // bg_kset_set_potential_ptr / bg_kset_band_density_sum buffers (lazily allocated)
  double** d_vts = nullptr;     // every operator's t.vt
  double* dens_part = nullptr;  // [k][chunk][grid]
  size_t dens_part_doubles = 0;
  double* dens_ksum = nullptr;  // [k][grid]
  size_t dens_ksum_doubles = 0;
  double* dens_w = nullptr;     // [k][column]
  size_t dens_w_doubles = 0;
  // bg_kset_sync: every operator's error word, gathered for one read
  int** d_errs = nullptr;
  int* d_errv = nullptr;
  int* h_errv = nullptr;
  bg::TcNl tc;  // tensor-core nonlocal products (BG_PREC_TENSOR)
};

namespace bg {
// Launch the local and nonlocal stages of operators [k0, k1) of a set on one stream
// (cols[k]: the widest block of operator k, used to size the grids).
// prec: BG_PREC_FP64, BG_PREC_FP32 or BG_PREC_TENSOR (tensor buffers sized beforehand
// by ensure_nonlocal_tc on tc, or on ks->tc when tc is null).
int enqueue_range(bg_kset* ks, int k0, int k1, const CallArgs* args, const int64_t* cols, cudaStream_t s,
                  StageEvents* ev, int prec = 0, TcNl* tc = nullptr);
// Convert the operator's potential to its FP32 copy on stream s if the copy is stale.
int ensure_potential_float(bg_op* op, cudaStream_t s);
// Failure message on the context (or the thread's context-free slot) and status.
int fail(bg_ctx* ctx, int code, const std::string& msg);
int cuda_fail(bg_ctx* ctx, cudaError_t e, const char* what);
// y = H x for a dense operator (device pointers, op stream).
int dense_apply(bg_op* op, const double* x, double* y, int64_t cols);
}  // namespace bg
