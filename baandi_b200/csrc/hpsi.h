// Device-side layout of one Hamiltonian operator (one k point) and the launchers of
// the H.x pipeline.  Shared by the CUDA kernels and the host runtime.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "fft_dev.cuh"

namespace bg {

// Immutable per-operator tables, resident in HBM.  The FFT box is n0 x n1 x n2
// (C order, z fastest).  Plane waves sit on S "sticks" (lines along z at fixed x, y);
// sticks are numbered so that a stick and its mirror (-x, -y) are adjacent and fall
// in the same group of at most `sg` sticks.
struct OpTables {
  int gamma;      // 1: real ORC rows, two columns per complex FFT
  int rows;       // npw (complex) or n ORC rows (Gamma)
  int S;          // sticks
  int ngroups;    // stick groups
  int nxact;      // x rows of the plane holding at least one stick
  int yper;       // x rows per warp in the 8-warp plane kernels' y passes
  int yper16;     // the same for the 16-warp plane kernels (one block per SM)
  const int* grp_stick;   // ngroups+1: first stick of each group
  const int* grp_entry;   // ngroups+1: entry range of each group
  const int2* entries;    // complex: (row g, pos); Gamma: (code, pos), code 0 for G=0,
                          // +(2i-1) at plus[i], -(2i-1) at minus[i]; pos = local stick * ld2 + z
  const int* grp_rep;     // Gamma: ngroups+1 representative range of each group
  const int4* reps;       // Gamma: (ORC row 2i-1 or 0, pos of plus, pos of minus, 0)
  const int* stick_plane; // S: x * pitch + y, offset inside the shared-memory plane
  const int* xact;        // nxact x rows
  const int* line_stick;  // nxact x n1: stick at (xact[i], y), -1 where the plane has none
  unsigned xbits[4];      // bit x set for every x row in xact (n0 <= 128)
  const double* kinetic;  // rows
  const double* vt;       // V(r) transposed to [z][y][x]
  const float* vtf;       // the same in FP32 (the FP32 apply), plane stride BoxGeo::vstridef
  double2* sbuf;          // stick buffer [unit][z][S]
  int* err;               // device error word (bit 0: non-finite input)
};

// Shape of the FFT box shared by every operator of one launch.
struct BoxGeo {
  int n0, n1, n2;
  int ld2;     // stride of a z line in the stick kernels' shared memory (odd)
  int pitch;   // row pitch of the shared-memory plane (odd)
  int sg;      // max sticks per group
  int vstride; // doubles between z planes of the transposed potential (even: 16-byte aligned planes)
  int vstridef; // floats between z planes of the FP32 potential (multiple of 4: 16-byte aligned planes)
  double inv_n;
  FftPlan p0, p1, p2;
  const double2* tw0;  // exp(+2 pi i q/n0), q < n0
  const double2* tw1;
  const double2* tw2;
  const float2* tw0f;  // FP32 copies (rounded from the same long double values)
  const float2* tw1f;
  const float2* tw2f;
};

// Block of one operator whose columns are decided on the device (a solver's correction
// block): kernels read x, y and the column count from here when CallArgs::dyn is set.
struct DynCols {
  const double* x;
  double* y;
  int cols;
  int units;
};

// Per-call arguments of one operator.
struct CallArgs {
  const double* x;  // complex: interleaved; Gamma: real ORC
  double* y;
  int64_t ldx, ldy; // column strides in doubles
  int cols;         // complex columns or real ORC columns
  int units;        // complex columns or column pairs
  const double* vt = nullptr;  // potential in the layout of OpTables::vt; nullptr: the operator's own
  int accumulate = 0;          // 1: y += FFT(V IFFT(scatter x))/N, no kinetic term (potential change)
  const DynCols* dyn = nullptr;  // device-side x, y, cols, units (grids sized for `cols`/`units`)
};

// The arguments with a device-side block resolved.
__device__ __forceinline__ CallArgs resolve(const CallArgs& in) {
  CallArgs a = in;
  if (a.dyn) {
    a.x = a.dyn->x;
    a.y = a.dyn->y;
    a.cols = a.dyn->cols;
    a.units = a.dyn->units;
  }
  return a;
}

// One launch covers up to kMaxBatch operators (k points) of the same grid; operator
// b of a launch works on blockIdx.z (local passes) with its own tables and blocks.
constexpr int kMaxBatch = 64;
struct Batch {
  int nk;
  CallArgs a[kMaxBatch];
};

// Nonlocal operands of one operator.
struct NlDev {
  const double* p;        // complex: 2*npw*nproj interleaved col-major; Gamma: real ORC n*nproj
  double* part;           // split-K partials [ks][col][nproj] (complex: x2)
  double* wd;             // coupled projections [col][nproj] (complex: x2)
  const int* atom_off;    // natoms+1 projector column offsets
  const int* d_off;       // natoms coupling offsets
  const double* d;        // concatenated row-major D blocks
  int rows;
  // complex operators: the projector table as bf16 hi/lo panels of the tensor-core
  // products (gemm_tc.cuh): p_tn for P^H x (K = rows), p_nn for P W (K = nproj)
  const unsigned char* p_tn;
  const unsigned char* p_nn;
  int kt_tn, kt_nn;
};

struct NlShape {
  int nproj, natoms, maxch;
  int ksplit, kchunk;
};

// Optional CUDA-event timing of every stage of an apply (stage s brackets its
// launch between ev[2s] and ev[2s+1] on the launching stream).
constexpr int kStages = 6;  // sticks_inverse, planes, sticks_forward, project, couple, back
struct StageEvents {
  bool on = false;
  cudaEvent_t ev[2 * kStages] = {};
};

// Enqueue the local + kinetic part: y = gather(FFT(V IFFT(scatter x)))/N + T x.
// tabs: device array of b.nk operator tables.  Returns the number of launches.
int launch_local(const OpTables* tabs, int gamma, int max_groups, const BoxGeo& g, const Batch& b, cudaStream_t s,
                 StageEvents* ev, int fp32 = 0);
// The FP32 local apply needs a cubic box with a compile-time plan.
bool fp32_supported(const BoxGeo& g);
// x rows per warp for the y passes of the plane kernels (warps 8 or 16) on an n0 x n1
// plane with nlines x rows holding sticks (1 where no compile-time plan covers the plane).
int plane_lines_per_warp(int n0, int n1, int nlines, int warps = 8);
// Enqueue y += P (D (P^H x)) (complex) or y += P (D (P^T x)) (Gamma).
int launch_nonlocal(const NlDev* nl, int gamma, const NlShape& sh, int max_rows, const Batch& b, cudaStream_t s,
                    StageEvents* ev);

// Buffers of the tensor-core nonlocal products (precision form, complex operators):
// the product descriptors of a batch (2 kMaxBatch), the workspace of the products (the
// split x and coupled-projection panels, the split-K partial tiles) and an error word.
// Sized by ensure_nonlocal_tc before any launch (and before a graph capture).
struct TcNl {
  void* desc = nullptr;
  void* work = nullptr;
  size_t work_bytes = 0;
  int* err = nullptr;
  int ksplit = 1;
  void release();
};
int ensure_nonlocal_tc(TcNl* tc, int nk, int nproj, int max_cols, int max_rows);
// Enqueue y += P (D (P^H x)) with P^H x and P W as BF16x3 tensor-core products (the
// coupling D in FP64); complex operators only.
int launch_nonlocal_tc(const NlDev* nl, const NlShape& sh, int max_rows, int max_cols, const Batch& b, TcNl* tc,
                       cudaStream_t s, StageEvents* ev);

// Band densities of the blocks of a batch (k = 0 .. b.nk - 1, operator tables tabs[k]
// and their stick buffers): part[k][c][z][y n0 + x] = sum over the units of chunk c of
// block k (in unit order) of w |psi(r)|^2, psi the unscaled inverse transform (Gamma:
// w_a Re^2 + w_b Im^2 of a column pair).  weights: device array, block k's column
// weights at k wstride; `chunks` chunks of `per_chunk` units per block.
int launch_density(const OpTables* tabs, int gamma, int max_groups, const BoxGeo& g, const Batch& b,
                   const double* weights, int wstride, int per_chunk, int chunks, double* part, cudaStream_t s);
// out (= or +=) the per-k chunk sums of part / volume, k points in order; ksum: scratch of
// nk grids (the per-k sums).
void launch_density_reduce(const double* part, int nk, int chunks, const BoxGeo& g, double volume, int accumulate,
                           double* ksum, double* out, cudaStream_t s);
// out[i] = *err[i], then *err[i] = 0 (the operators' error words, read and cleared).
void launch_gather_errors(int* const* err, int n, int* out, cudaStream_t s);
// Copy n doubles from src to each of the ndst device pointers in dst (a device array).
void launch_broadcast(const double* src, int64_t n, double* const* dst, int ndst, cudaStream_t s);
void launch_potential_transpose(const double* v, const BoxGeo& g, double* vt, int* err, cudaStream_t s);
// vtf = (float) vt plane by plane (the FP32 apply's potential).
void launch_potential_float(const double* vt, const BoxGeo& g, float* vtf, cudaStream_t s);

// Radix plan of a line of n <= 128 points (2, 3, 4, 5) for fft_lines; false if n has
// another prime factor.  twiddles(n): exp(+2 pi i q/n), q < n, interleaved (re, im).
bool make_fft_plan(int n, FftPlan* p);
std::vector<double> twiddles(int n);

size_t plane_smem_bytes(const BoxGeo& g);
size_t stick_smem_bytes(const BoxGeo& g);
int configure_kernels(size_t plane_smem, size_t stick_smem);

}  // namespace bg
