// Complex products on the tcgen05 tensor cores with BF16x3 split operands and FP32
// accumulation: the precision form of the projector and subspace products.
//
//   kTN  C[M x N] (=, +=, -=) A^H B   A: K x M, B: K x N  (Gram products, projections)
//   kNN  C[M x N] (=, +=, -=) A B     A: M x K, B: K x N  (rotations, back-projection)
//
// All matrices are column-major complex (interleaved FP64).  Every FP64 value x is split
// into x_hi = bf16(x) and x_lo = bf16(x - x_hi); a product of two values is
// a_hi b_hi + a_hi b_lo + a_lo b_hi (the a_lo b_lo term, 2^-18 relative, is dropped), so
// each term carries about 16 significant bits before the FP32 accumulation.  The complex
// product is one real product of twice the depth and twice the width: K index 2k + p
// holds part p of element k, output column 2j + q part q of column j.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace bg {
namespace tc {

enum : int { kTN = 0, kNN = 1 };
enum : int { kStore = 0, kAdd = 1, kSub = 2 };

// One product (device pointers; M, N, K complex dimensions; M = 0 marks an empty slot).
struct ZDesc {
  const double2* A;
  const double2* B;
  double2* C;
  int64_t lda, ldb, ldc;
  int M, N, K;
  int op;  // kStore, kAdd, kSub
};

constexpr int kTileM = 128;        // MMA rows
constexpr int kTileN = 256;        // MMA columns (128 complex output columns)
constexpr int kStepK = 32;         // complex K per pipeline stage (64 real)

// Workspace (floats) of one kTN launch: ksplit partial tiles per descriptor.
inline size_t tn_workspace_floats(int ndesc, int ksplit, int max_m, int max_n) {
  return (size_t)ndesc * ksplit * (size_t)max_m * 2 * (size_t)max_n;
}

// Launches over `ndesc` device descriptors (d_desc in device memory).  max_m, max_n and
// max_k bound every descriptor's dimensions (they size the grid).  kTN: split-K with
// ksplit slices into `work` (tn_workspace_floats) and an ordered FP64 reduction;
// kNN: one slice, written straight into C.  err: device word, set to 1 when a bounded
// wait of the pipeline gives up.  Returns the number of launches.
int launch_zgemm(int mode, const ZDesc* d_desc, int ndesc, int max_m, int max_n, int max_k, int ksplit,
                 float* work, int* err, cudaStream_t s);

// A split count that gives about two waves of 148 SMs for a kTN product.
int tn_ksplit(int ndesc, int max_m, int max_n, int max_k);

// Shared-memory attributes (once per device).
cudaError_t prepare_zgemm();

}  // namespace tc
}  // namespace bg
