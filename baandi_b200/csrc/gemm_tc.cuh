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
//
// A product runs in two passes.  The split pass (memory bound) writes both operands as
// bf16 hi/lo panels in the order the MMA consumes them: a panel is a sequence of tiles
// (row tile rt, K tile kt) at (rt * kt_count + kt) * tile_bytes, each tile the hi block
// then the lo block of rows x 32 real K values in the canonical K-major layout without
// swizzle (8-row x 16-byte core matrices; K chunk c of row r at c * rows * 16 +
// (r / 8) * 128 + (r % 8) * 16 bytes).  The product pass streams whole tiles into
// shared memory with bulk copies and feeds them to tcgen05.mma.  A constant operand (the
// projector table) is split once (split_a) and named in ZDesc::a_split.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

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
  const unsigned char* a_split = nullptr;  // A as a panel from split_a (then A is not read)
  int a_kt = 0;                            // K tiles of that panel (k_tiles(K) of its split)
};

constexpr int kTileM = 128;     // MMA rows (A tile rows)
constexpr int kTileNMax = 256;  // MMA columns at most (B tile rows: 128 complex output columns)
constexpr int kStepK = 32;      // real K values per tile (16 complex)

// K tiles of a K-complex-deep operand.
inline int k_tiles(int64_t k) { return (int)((2 * k + kStepK - 1) / kStepK); }
// Bytes of a tile of `rows` rows (hi and lo blocks).
inline size_t tile_bytes(int rows) { return (size_t)rows * kStepK * 2 * 2; }
// B tile rows of a launch whose products have at most max_n complex columns.
inline int b_tile_rows(int max_n) {
  const int r = (2 * max_n + 15) / 16 * 16;
  return r < kTileNMax ? r : kTileNMax;
}
// Bytes of a panel of A with `rows` MMA rows (kTN: M; kNN: M) and K complex depth.
inline size_t a_panel_bytes(int rows, int64_t k) {
  return (size_t)((rows + kTileM - 1) / kTileM) * (size_t)k_tiles(k) * tile_bytes(kTileM);
}

// Workspace (bytes) of one launch: the split panels of every descriptor (A's only when
// a_presplit is false) and, for kTN, the ksplit FP32 partial tiles per descriptor.
size_t workspace_bytes(int mode, int ndesc, int max_m, int max_n, int max_k, int ksplit, bool a_presplit);

// Launches over `ndesc` device descriptors (d_desc in device memory): the split pass and
// the product (kTN: split K with ksplit slices and an ordered FP64 reduction of the FP32
// partial tiles; kNN: one slice, written straight into C).  max_m, max_n and max_k bound
// every descriptor's dimensions (they size the grids and the workspace); a_presplit:
// every non-empty descriptor names its A panel.  err: device word, set to 1 when a
// bounded wait of the pipeline gives up.  Returns the number of launches.
int launch_zgemm(int mode, const ZDesc* d_desc, int ndesc, int max_m, int max_n, int max_k, int ksplit,
                 bool a_presplit, void* work, int* err, cudaStream_t s);

// A split count that fills whole waves of 148 SMs for a kTN product (at most 4,096 complex
// K per split).
int tn_ksplit(int ndesc, int max_m, int max_n, int max_k);

// The autotuner's split count for a kTN product of these bounds: the candidates that fill
// whole waves (from the accuracy bound's minimum) timed once per shape on scratch panels
// (product pass and reduction, CUDA events on a private stream, best of two after a warm
// launch), the fastest kept for the process; the rule's count when a measurement fails.
// Synchronous; never call it inside a stream capture.
int tn_ksplit_tuned(int ndesc, int max_m, int max_n, int max_k);

// The tuner's decisions so far as a JSON array.
std::string tuning_report();

// Writes A of a `mode` product (kTN: K x M, kNN: M x K, ld lda) as a panel of
// a_panel_bytes(M, K) bytes (K tiles: k_tiles(K)).
cudaError_t split_a(int mode, const double2* A, int64_t lda, int M, int K, unsigned char* panel, cudaStream_t s);

// Shared-memory attributes (once per device).
cudaError_t prepare_zgemm();

}  // namespace tc
}  // namespace bg
