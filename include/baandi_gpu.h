/* baandi_gpu.h -- C ABI of the B200 Hamiltonian-apply library (libbaandi_b200.so).
 *
 * The library applies the Kohn-Sham Hamiltonian H = T + V_loc(r) + V_NL to blocks of
 * plane-wave coefficient columns on one GPU, and builds the operands of that apply.
 * Every entry point returns an int status: BG_OK (0) or one of the BG_E* codes below;
 * bg_last_error() gives the message of the last failure on a context.
 *
 * Layouts.  Coefficient blocks are column-major, one column per band.  Complex values
 * are interleaved (re, im) doubles.  The local potential is the full real grid in C
 * order, flat index (i*n1 + j)*n2 + k for grid point r = i/n0 a1 + j/n1 a2 + k/n2 a3.
 *
 * Each operator mirrors one reference Hamiltonian (paths inside the reference project):
 *   complex (k point)  crates/dft-physics/src/distributed_complex.rs:58-386
 *                      (trait DistributedComplexOperator, crates/dft-solvers/src/
 *                      ref_davidson_complex.rs:41-56)
 *   real Gamma (ORC)   crates/dft-physics/src/distributed_real_gamma.rs:120-1352
 *                      (trait DistributedRealOperator, crates/dft-solvers/src/
 *                      distributed_davidson.rs:23-40)
 * with one rank: the communicator argument of the reference calls has no counterpart.
 */
#ifndef BAANDI_GPU_H
#define BAANDI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- status codes */
#define BG_OK 0
#define BG_ESHAPE 1     /* dimensions, row/column counts or layout mismatch        */
#define BG_ENONFINITE 2 /* a NaN or infinity in an input                           */
#define BG_EEPOCH 3     /* potential epoch not strictly increasing / never set     */
#define BG_EDEVICE 4    /* CUDA runtime or kernel failure                          */
#define BG_ETIMEOUT 5   /* a bounded device wait gave up                           */
#define BG_EINVAL 6     /* invalid argument (null pointer, bad option)            */
#define BG_ENOMEM 7     /* device or host allocation failed                        */

/* pointer kinds of bg_op_apply_block */
#define BG_PTR_HOST 0   /* synchronous: copies in, applies, copies out, validates   */
#define BG_PTR_DEVICE 1 /* asynchronous on the operator's stream                    */

/* arithmetic of bg_op_apply_block: FP64, or the precision form with the local part
 * (scatter, 3D transforms, x V(r), gather) in FP32 on the element stream and the
 * kinetic and nonlocal parts in FP64; blocks stay FP64 in memory.  FP32 needs a cubic
 * grid of 25, 45, 54, 60, 72 or 108 points. */
#define BG_PREC_FP64 0
#define BG_PREC_FP32 1
#define BG_PREC_TENSOR 2  /* FP32 local part; P^H x and P W as BF16x3 tensor-core
                             products (complex operators; a Gamma-real operator keeps
                             its nonlocal part in FP64) */

typedef struct bg_ctx bg_ctx;
typedef struct bg_op bg_op;

typedef struct {
  int32_t device;       /* CUDA ordinal */
  int32_t reserved[7];  /* zero */
} bg_device_opts;

/* --------------------------------------------------------------------- context */
int bg_ctx_create(const bg_device_opts* opts, bg_ctx** out);
int bg_ctx_destroy(bg_ctx* ctx);
/* Copies the last failure message of `ctx` (or of context-free calls when ctx is
 * NULL) into buf, NUL-terminated, truncated to len. */
int bg_last_error(const bg_ctx* ctx, char* buf, size_t len);

/* ------------------------------------------------------------------- operators */
/* Plane-wave basis of one k point.  miller: npw integer triples (G = sum m_j b_j),
 * in the caller's row order; kinetic: 1/2 |k+G|^2 (Ha) per row; dims: FFT grid.
 * k != 0 maps Miller indices modulo the grid; at Gamma they must lie in the
 * canonical interval [-n/2, (n-1)/2] (crates/dft-basis/src/lib.rs:380-398, 491-502). */
typedef struct {
  int64_t npw;
  const int32_t* miller;
  const double* kinetic;
  int32_t dims[3];
  int32_t gamma; /* 1: exactly Gamma (canonical-interval check applies) */
} bg_basis_desc;

/* Nonlocal projectors: table is column-major npw x nproj complex (interleaved), the
 * reference's beta(k+G) columns (crates/dft-physics/src/hamiltonian.rs:2605-2760);
 * channels[a] columns belong to atom a, in order; couplings are the per-atom
 * channels[a] x channels[a] row-major D blocks (Ha), concatenated. */
typedef struct {
  int32_t nproj;
  const double* table;
  int32_t natoms;
  const int32_t* channels;
  const double* couplings;
} bg_projectors;

/* Replaces DistributedComplexHamiltonian::new_owned (distributed_complex.rs:88-167)
 * with one rank.  capacity = widest block bg_op_apply_block accepts. */
int bg_op_create_complex(bg_ctx* ctx, const bg_basis_desc* basis, const bg_projectors* proj,
                         int64_t capacity, bg_op** out);

/* Replaces DistributedRealHamiltonian::new_owned (distributed_real_gamma.rs:228-247,
 * from_parts :249-420) with one rank.  `basis` is the full Gamma sphere (row 0 = G=0,
 * every -G present); `proj` its complex table; rows of the operator are the ORC rows
 * of crates/dft-basis/src/half.rs:31-37 (n = npw real rows). */
int bg_op_create_gamma_real(bg_ctx* ctx, const bg_basis_desc* basis, const bg_projectors* proj,
                            int64_t capacity, bg_op** out);

int bg_op_destroy(bg_op* op);

/* Replaces set_owned_potential (distributed_complex.rs:252-264): v is the full real
 * grid (n0*n1*n2, C order, host memory); epoch must exceed the previous one. */
int bg_op_set_potential(bg_op* op, const double* v_grid, uint64_t epoch);

/* Replaces apply_block (distributed_complex.rs:340-386; distributed_real_gamma.rs:
 * 1062-1264): y = H x, y completely overwritten.  rows must equal the operator's row
 * count (npw), 0 <= cols <= capacity.  Complex operators take interleaved complex
 * columns, the Gamma operator real ORC columns.  ptr_kind BG_PTR_HOST: synchronous;
 * a non-finite x returns BG_ENONFINITE (y is then unspecified).  BG_PTR_DEVICE:
 * enqueued on the operator's stream, a non-finite x is reported by bg_op_sync; x must
 * not alias y. */
int bg_op_apply_block(bg_op* op, const double* x, double* y, int64_t rows, int64_t cols,
                      int32_t ptr_kind, int32_t precision);

/* Kinetic plus nonlocal diagonal T_g + sum D_ij Re(P_gi conj(P_gj)) per row (Ha),
 * the reference's static_diagonal (distributed_complex.rs:29-53); host buffer of
 * `rows` doubles (ORC order for the Gamma operator). */
int bg_op_diagonal(const bg_op* op, double* out);

/* Row count (global_len), capacity, and the operator's CUDA stream (cudaStream_t). */
int bg_op_rows(const bg_op* op, int64_t* rows);
int bg_op_capacity(const bg_op* op, int64_t* capacity);
int bg_op_stream(const bg_op* op, void** stream);
/* Use the caller's stream (cudaStream_t, e.g. a torch stream) for BG_PTR_DEVICE work. */
int bg_op_set_stream(bg_op* op, void* stream);
/* Wait for the operator's stream and report a device error recorded by earlier
 * BG_PTR_DEVICE applies (BG_ENONFINITE for a non-finite input column). */
int bg_op_sync(bg_op* op);
/* Count of this library's kernel launches issued by the operator so far. */
int bg_op_launches(const bg_op* op, int64_t* launches);

/* Per-stage CUDA-event timing (tracing): when enabled, every apply records events
 * around its six launches (sticks_inverse, planes, sticks_forward, project, couple,
 * back); stage_times waits for the stream and returns the last apply's stage times in
 * milliseconds (ms[6]). */
int bg_op_profile(bg_op* op, int32_t enable);
int bg_op_stage_times(bg_op* op, double* ms);

/* ------------------------------------------------------------ SCF map steps */
/* set_owned_potential with the grid given by pointer kind: BG_PTR_HOST is
 * bg_op_set_potential; BG_PTR_DEVICE takes a C-order grid in device memory, checks it
 * on the device and returns BG_ENONFINITE (old potential kept) before installing it. */
int bg_op_set_potential_ptr(bg_op* op, const double* v_grid, uint64_t epoch, int32_t ptr_kind);

/* Replaces add_local_change (distributed_complex.rs:388-420; the Gamma form is
 * distributed_real_gamma.rs:1370-1430 followed by the sum of
 * crates/dft-engine/src/refscf/kept_hx.rs:98-160): hx += FFT(change(r) IFFT(x))/N, the
 * kept-HX update H_new x = H_old x + (V_new - V_old) x, no kinetic or nonlocal term.
 * change is a C-order grid (n0*n1*n2), x and hx blocks as in bg_op_apply_block, all
 * three of the same pointer kind.  A non-finite change returns BG_ENONFINITE before
 * hx is touched.  A non-finite x or hx: BG_PTR_HOST returns BG_ENONFINITE and leaves
 * the caller's hx unchanged; BG_PTR_DEVICE reports it at bg_op_sync (hx unspecified). */
int bg_op_add_local_change(bg_op* op, const double* x, const double* change, double* hx,
                           int64_t rows, int64_t cols, int32_t ptr_kind);

/* Replaces band_density_sum (distributed_complex.rs:485-547; Gamma ORC columns:
 * distributed_real_gamma.rs:744-785): density(r) = sum_b weights[b] |psi_b(r)|^2 /
 * volume over the cols columns of x in band order, psi_b the unscaled inverse
 * transform sum_G x_bG e^{iGr} (Gamma: the real function of ORC column b).  density is
 * a C-order grid (n0*n1*n2), overwritten (accumulate 0) or added to (accumulate 1:
 * the k-point sum of a map).  weights (host, cols values) must be finite and >= 0,
 * volume finite and > 0 (BG_ESHAPE).  x and density have the pointer kind; a
 * non-finite x is reported like bg_op_apply_block's. */
int bg_op_band_density_sum(bg_op* op, const double* x, int64_t rows, int64_t cols,
                           const double* weights, double volume, double* density,
                           int32_t accumulate, int32_t ptr_kind);

/* ------------------------------------------------------------ fields of a map */
/* Hartree and LDA-PZ fields of a density on the FFT box, the field step of a map
 * (crates/dft-engine/src/refscf/map.rs:41-198 with LDA-PZ, crates/dft-physics/src/
 * xc.rs:39-77).  A fields object holds the box (lattice vectors as the ROWS of rows[9],
 * Bohr; dims 2,3,5-smooth, each at most 128), its transforms and work grids. */
typedef struct bg_fields bg_fields;
int bg_fields_create(bg_ctx* ctx, const double rows[9], const int32_t dims[3], bg_fields** out);
int bg_fields_destroy(bg_fields* f);
/* Use the caller's stream (cudaStream_t) for the field kernels. */
int bg_fields_set_stream(bg_fields* f, void* stream);
/* Cell volume (Bohr^3) of the box. */
int bg_fields_volume(const bg_fields* f, double* volume);
/* density (C-order grid, signed) -> v_hxc = V_H + v_xc and V_H (v_h may be NULL) on
 * the same grid: rho(G) = to_reciprocal(density) (1/N), V_H(G) = 4 pi rho(G) / |G|^2
 * with V_H(0) = 0 and G from the canonical Miller index of every grid point,
 * V_H(r) = Re sum_G V_H(G) e^{iGr}; v_xc = LDA-PZ of |density| (0 at or below 1e-10).
 * energies (host, 3 values, Ha): dV/2 sum rho V_H, dV sum |rho| eps_xc, dV sum rho v_xc.
 * density, v_hxc and v_h have the pointer kind; the call returns when the energies
 * are on the host.  A non-finite density value returns BG_ENONFINITE. */
int bg_fields_lda_hartree(bg_fields* f, const double* density, double* v_hxc, double* v_h,
                          double energies[3], int32_t ptr_kind);
/* The mixer's coefficient space (crates/dft-engine/src/refscf/density.rs:27-237): the
 * half sphere of the density basis, given once as n flat C-order grid indices (host).
 * sphere_forward: coeffs[i] = FFT(density)/N at index i (complex, interleaved);
 * sphere_inverse: density = 2 Re(sum_i c_i e^{iG_i r}) - Re c_0 (the inverse of the
 * positive half alone).  Both synchronous; arrays have ptr_kind. */
int bg_fields_set_sphere(bg_fields* f, int64_t n, const int64_t* flat_index);
int bg_fields_sphere_forward(bg_fields* f, const double* density, double* coeffs, int32_t ptr_kind);
int bg_fields_sphere_inverse(bg_fields* f, const double* coeffs, double* density, int32_t ptr_kind);

/* ------------------------------------------------------------ density mixing */
/* The reference mixer (crates/dft-engine/src/refscf/broyden.rs, metric.rs) on the GPU:
 * an unnormalised difference-history Anderson update of complex reciprocal-space
 * vectors of n entries (interleaved doubles) under the Hartree metric
 * w_G = 8 pi metric_volume / G^2 on smooth G != 0 (0 elsewhere), Ry. */
typedef struct bg_mixer bg_mixer;
typedef struct {
  double beta;           /* (0, 1], reference default 0.7                              */
  int32_t history;       /* 1..25, reference default 8                                 */
  int32_t thomas_fermi;  /* nonzero: screen F~ by G^2 / (G^2 + a) on smooth G         */
  int32_t reserved[4];
} bg_mixer_profile;
typedef struct {
  int32_t iteration;     /* updates so far, this one included                          */
  int32_t occupancy;     /* secant pairs used                                          */
  int32_t inserted_slot; /* ring slot written by this update, -1 on the first          */
  int32_t reserved;
  double gamma_l2, gamma_max;
  double condition;      /* lambda_max / lambda_min of the history Gram (0: no history) */
} bg_mixer_diagnostics;
/* g2: n values |G|^2 (Bohr^-2), smooth: n flags; volume and electrons set the Thomas-
 * Fermi wave number (broyden.rs:96-123); metric_volume the metric weights. */
int bg_mixer_create(bg_ctx* ctx, const bg_mixer_profile* profile, int64_t n, const double* g2,
                    const int32_t* smooth, double volume, double electrons, double metric_volume,
                    bg_mixer** out);
int bg_mixer_destroy(bg_mixer* m);
int bg_mixer_set_stream(bg_mixer* m, void* stream);
/* Broyden::update (broyden.rs:319-435): next from x and F = y - x.  A numerically
 * rank-deficient history (lambda_min <= p eps lambda_max) returns BG_EINVAL ("singular
 * Broyden history ...") and, like a non-finite result (BG_ENONFINITE), ends the mixer:
 * later updates fail.  Returns when next is ready (x, f, next have ptr_kind). */
int bg_mixer_update(bg_mixer* m, const double* x, const double* f, double* next, int32_t ptr_kind,
                    bg_mixer_diagnostics* diag);
/* gamma of the last update (host, up to 25 values; *count = its occupancy). */
int bg_mixer_gamma(const bg_mixer* m, double* gamma, int32_t* count);
/* F~ = F - gamma.dF of the last update before screening (broyden.rs:200-206). */
int bg_mixer_reduced_residual(bg_mixer* m, double* out, int32_t ptr_kind);
/* The metric form <a, b> (metric.rs:147-200), Ry. */
int bg_mixer_metric(bg_mixer* m, const double* a, const double* b, double* out, int32_t ptr_kind);

/* ------------------------------------------------------------ k-point sets */
/* All bands of several k points in one launch per stage.  The reference solves the k
 * points of a map one after another (crates/dft-engine/src/refscf/k_map.rs:136-210,
 * each calling apply_block of its own DistributedComplexHamiltonian); a set keeps
 * each operator's tables and applies every operator's block in one batched launch.
 * Operators must share the context, grid, kind and projector layout; 1..64 of them.
 * The set borrows the operators: destroy it before them. */
typedef struct bg_kset bg_kset;
int bg_kset_create(bg_ctx* ctx, int32_t n, bg_op* const* ops, bg_kset** out);
int bg_kset_destroy(bg_kset* set);
/* y[k] = H_k x[k] for every operator k of the set (cols[k] columns, 0 allowed);
 * pointer kinds and precision as bg_op_apply_block. */
int bg_kset_apply(bg_kset* set, const double* const* x, double* const* y, const int64_t* cols,
                  int32_t ptr_kind, int32_t precision);
/* The potential of every operator of the set from one C-order grid: the per-k install
 * of bg_op_set_potential_ptr (the reference installs V in each k point's Hamiltonian,
 * crates/dft-engine/src/refscf/k_map.rs:136-210 with map.rs:200-260) done once for the
 * set: transposed and checked once (one wait; a non-finite grid leaves every operator's
 * potential as it was, BG_ENONFINITE), then copied to each operator on the set's
 * stream.  epoch must exceed every operator's.  BG_PTR_HOST installs per operator. */
int bg_kset_set_potential_ptr(bg_kset* set, const double* v, uint64_t epoch, int32_t ptr_kind);
/* density (= or, accumulate != 0, +=) sum over the set's k points of
 * bg_op_band_density_sum(k, x[k], cols, weights + k cols, volume): the k-summed band
 * density of a map (reference k_map.rs:136-210 with band_density_sum,
 * crates/dft-physics/src/distributed_complex.rs:485-547) in one batched launch per
 * stage, k points added in order.  Device blocks (layout of bg_kset_apply) and device
 * grid (BG_PTR_DEVICE only); weights on the host, n_k x cols, finite and >= 0. */
int bg_kset_band_density_sum(bg_kset* set, const double* const* x, int64_t cols, const double* weights,
                             double volume, double* density, int32_t accumulate, int32_t ptr_kind);
int bg_kset_sync(bg_kset* set);
int bg_kset_stream(const bg_kset* set, void** stream);
int bg_kset_set_stream(bg_kset* set, void* stream);
int bg_kset_launches(const bg_kset* set, int64_t* launches);
int bg_kset_profile(bg_kset* set, int32_t enable);
int bg_kset_stage_times(bg_kset* set, double* ms);

/* ------------------------------------------------------------ block Davidson */
/* Options and Solution mirror crates/dft-solvers/src/ref_davidson.rs:39-93. */
typedef struct {
  int64_t bands;          /* n: lowest eigenpairs wanted                                 */
  double threshold;       /* occupied Ritz-change threshold (Ha, strict inequality)       */
  int64_t occupied;       /* leading occupied bands; others use max(5 threshold, 5e-6)   */
  int32_t first_step;     /* nonzero: every band uses `threshold`                       */
  int64_t capacity;       /* basis columns; 0 selects min(rows, 2 bands)                 */
  int32_t max_iterations; /* correction iterations (reference default 20)               */
  int32_t flags;          /* bg_kset_davidson_solve: bit 0 launches directly (no graph)  */
  int32_t preconditioner; /* BG_PRECOND_*                                                */
  int32_t apply_precision; /* BG_PREC_* of the solver's H applies; BG_PREC_TENSOR in
                              bg_kset_davidson_solve is the precision form: a first phase
                              with tensor-core applies, H Grams and rotations (overlap
                              Grams, factor and eigensolve FP64) until every active band's
                              residual |HX_j - lambda_j X_j| is below 1e-4 (or stops
                              falling), then the FP64 solve from its Ritz vectors
                              (convergence judged in FP64); a tensor phase that converges
                              every band by the Ritz-change criterion ends the solve */
  int32_t reserved[1];
} bg_davidson_options;

/* Correction of band j from its residual r = HX_j - lambda_j X_j on row g (the
 * Preconditioner seam, crates/dft-solvers/src/lib.rs:83-102, and its variants
 * :176-207, real_davidson.rs:1130-1170):
 *   BG_PRECOND_SMOOTH      r / d(h_g, lambda_j), the reference Davidson's smooth
 *                          denominator (ref_davidson.rs:418-422); diagonal = H diagonal
 *   BG_PRECOND_TPA         -r tpa(t_g, s_j) with s_j = max(0.1, sum |X_gj|^2 t_g /
 *                          sum |X_gj|^2) (lib.rs:176-206); diagonal = kinetic t_g
 *   BG_PRECOND_RITZ_SHIFT  -r / max(h_g - lambda_j, 0.1); diagonal = H diagonal
 *   BG_PRECOND_LEARNED     -r tpa(t_g, s_j) exp(clamp(m(f_gj), -3, 3)), m the context's
 *                          per-G network (bg_learned_set) on f = (log max(t_g/s_j, 1e-4),
 *                          log(t_g + 0.05), log s_j, lambda_j, log(|r_g| / rms_j r));
 *                          diagonal = kinetic t_g.  bg_davidson_solve only.  The solve
 *                          falls back to TPA (stats.fallbacks = 1) once the largest Ritz
 *                          change has not fallen below its best for 5 iterations or half
 *                          of max_iterations is spent. */
#define BG_PRECOND_SMOOTH 0
#define BG_PRECOND_TPA 1
#define BG_PRECOND_RITZ_SHIFT 2
#define BG_PRECOND_LEARNED 3

typedef struct {
  int32_t iterations;
  int32_t reduced_solves;
  int64_t h_calls;
  int64_t h_columns;
  int32_t repairs;
  int32_t contractions;
  int32_t dropped;         /* corrections dropped as dependent or of vanishing norm     */
  int32_t converged_count;
  int32_t fallbacks;       /* 1: the learned preconditioner gave way to TPA in this solve */
  int32_t tensor_iterations; /* BG_PREC_TENSOR: iterations before the FP64 handover       */
} bg_davidson_stats;

/* Reference block Davidson (crates/dft-solvers/src/ref_davidson.rs:117-366 for the
 * Gamma operator, ref_davidson_complex.rs:641-1110 for complex operators): H applies
 * and subspace products on the GPU, the reduced problem on the host.  start: rows x
 * bands column-major host block (interleaved complex for complex operators);
 * diagonal: rows host doubles (kinetic + nonlocal diagonal + mean local potential).
 * Outputs (host): eigenvalues[bands] ascending, eigenvectors rows x bands, converged
 * flags (Ritz change below the band threshold).  An iteration limit returns BG_OK
 * with unconverged flags, as the reference does.  The operator's capacity must be at
 * least the Davidson capacity. */
int bg_davidson_solve(bg_op* op, const double* start, const double* diagonal,
                      const bg_davidson_options* options, double* eigenvalues, double* eigenvectors,
                      int32_t* converged, bg_davidson_stats* stats);

/* The same reference Davidson for every k point of a set at once, driven from the GPU
 * (the reference solves the k points of a map one after another,
 * crates/dft-engine/src/refscf/k_map.rs:136-210, each with ref_davidson_complex.rs:
 * 798-1082).  Every large product is one launch over all k points, the reduced problem
 * (bordered Cholesky, Householder tridiagonalisation, tridiagonal eigenpairs) and the
 * control decisions (contraction, dropped corrections, repair, convergence) run in a
 * one-block-per-k-point kernel -- at capacities 129 .. 1152 the factor and the eigensolve
 * run on many blocks (cooperative launches, bg_reduced_eigh) -- and one iteration is a CUDA
 * graph replayed until all k points finish.  Per-k arrays (nk = set size): start[k] rows_k x bands, diagonal[k]
 * rows_k, eigenvalues[k] bands, eigenvectors[k] rows_k x bands, converged[k] bands;
 * start/diagonal/eigenvectors have ptr_kind (eigenvalues and converged are host);
 * stats: nk entries or NULL.  options.flags bit 0 set: launch the iteration's
 * kernels directly instead of replaying the graph (same results); bit 1: the reduced
 * problem on many blocks at any capacity; bit 2: on the one-block control kernel at any
 * capacity.  The Davidson
 * capacity is the smallest over the k points; bands must fit every operator's capacity.
 * Errors name the k point; the solve runs on the set's stream and returns when done. */
int bg_kset_davidson_solve(bg_kset* set, const double* const* start, const double* const* diagonal,
                           const bg_davidson_options* options, int32_t ptr_kind, double* const* eigenvalues,
                           double* const* eigenvectors, int32_t* const* converged, bg_davidson_stats* stats);

/* Replaces solve_with_initial_hx (crates/dft-solvers/src/ref_davidson_complex.rs:641) as the
 * SCF's kept-HX path uses it (crates/dft-engine/src/refscf/kept_hx.rs:98-160): the same
 * solve as bg_kset_davidson_solve with device blocks only, where start_hx (NULL, or one
 * rows x bands block per k point) holds H applied to the start block (kept from the
 * previous solve and brought to the current potential with bg_op_add_local_change), so the
 * start needs no apply, and eigenvectors_hx (NULL, or one block per k point) receives H
 * applied to the returned eigenvectors.  With the precision form, eigenvectors_hx carries
 * the final phase's precision (FP64 unless the tensor phase ended the solve:
 * stats.tensor_iterations == stats.iterations); the FP64 phase after a handover applies H
 * itself. */
int bg_kset_davidson_solve_hx(bg_kset* set, const double* const* start, const double* const* start_hx,
                              const double* const* diagonal, const bg_davidson_options* options,
                              double* const* eigenvalues, double* const* eigenvectors, double* const* eigenvectors_hx,
                              int32_t* const* converged, bg_davidson_stats* stats);

/* The autotuner's decisions so far (the split-K counts of the tensor-core A^H B products,
 * timed once per shape when a precision-form apply or solve first needs them) as a JSON
 * array with the measured times: written to buf (capacity bytes, NUL-terminated,
 * truncated to fit); returns the bytes the whole report needs. */
int bg_autotune_report(char* buf, int64_t capacity);

/* The generalised Hermitian eigenproblem H C = S C diag(w) of one m x m pencil (m <=
 * 1152; column-major host matrices, interleaved complex when is_complex), solved the way
 * bg_kset_davidson_solve solves its reduced problem beyond capacity 128: the Cholesky
 * factor of S with the reference's pivot rule (squared pivot over the overlap diagonal
 * >= eps / 1e-12, crates/dft-solvers/src/lean_davidson.rs:62-70), A = L^-1 H L^-H, a
 * Householder tridiagonalisation, bisection and inverse iteration, C = L^-H Y -- the
 * reference's ComplexOverlapFactor::extend + solve_lowest_into
 * (crates/dft-numerics/src/linalg.rs:276, :369) -- on many thread blocks of the
 * context's device.  Outputs (host): all m eigenvalues ascending and the S-orthonormal
 * eigenvectors (m x m).  device_ms (may be NULL): device time of the solve.  A
 * dependent S returns BG_ESHAPE. */
int bg_reduced_eigh(bg_ctx* ctx, int64_t m, int32_t is_complex, const double* s, const double* h,
                    double* eigenvalues, double* vectors, double* device_ms);

/* Complex product on the tcgen05 tensor cores with BF16x3 split operands and FP32
 * accumulation (the precision form's projector and subspace products; no counterpart
 * in the reference, whose products are FP64 faer/MKL GEMMs, crates/dft-physics/src/
 * distributed_complex.rs:284-338, crates/dft-solvers/src/ref_davidson_complex.rs:195,
 * :277).  mode 0: C (op)= A^H B with A k x m, B k x n; mode 1: C (op)= A B with A m x k,
 * B k x n.  op 0: C = product, 1: C += product, 2: C -= product.  Device pointers,
 * column-major interleaved complex FP64 with leading dimensions in complex elements.
 * Each FP64 value is split into bf16 hi + lo; a product keeps hi*hi + hi*lo + lo*hi, so
 * an entry's error is about 1e-5 of sum_r |a_r| |b_r| (16 significant bits, FP32
 * accumulation).  Runs on `stream` and returns when done (it allocates its split-K
 * workspace per call). */
int bg_zgemm_bf16x3(bg_ctx* ctx, int32_t mode, int64_t m, int64_t n, int64_t k, const double* a, int64_t lda,
                    const double* b, int64_t ldb, double* c, int64_t ldc, int32_t op, void* stream);

/* Dense operator y = H x of a rows x rows column-major matrix (interleaved complex when
 * is_complex), for fixtures and small exact tests of the solver. */
int bg_op_create_dense(bg_ctx* ctx, int64_t rows, const double* h, int32_t is_complex, int64_t capacity,
                       bg_op** out);

/* ------------------------------------------------------------ learned preconditioner */
/* No counterpart in the reference (its Preconditioner seam, crates/dft-solvers/src/
 * lib.rs:83-102, takes any correction; TPA is :176-207).  A per-G-vector network
 * 5 -> 64 -> 64 -> 1 (GELU) with BF16 parameters and FP32 accumulation; its output m is
 * a log-multiplier on the TPA factor (BG_PRECOND_LEARNED).  Parameter layout, one array of
 * BG_LEARNED_PARAMS: W1 [64][5], b1 [64], W2 [64][64] (row = output), b2 [64], w3 [64],
 * b3.  A network with w3 = 0 and b3 = 0 is exactly TPA. */
#define BG_LEARNED_PARAMS 4609

/* The context's network for BG_PRECOND_LEARNED: host FP32 parameters, rounded to BF16
 * (nearest even) and copied to the device; non-finite parameters are rejected. */
int bg_learned_set(bg_ctx* ctx, const float* params);
int bg_learned_clear(bg_ctx* ctx);

/* Training samples (device arrays of n entries; one sample per (row g, band j)):
 * feats n x 5 inputs, base the TPA factor -tpa(t_g, s_j), a = |r_g|^2, z = conj(r_g) e_g
 * (n interleaved complex floats), col the band's column; ecol[ncols] = |e_j|^2. */
typedef struct {
  int64_t n;
  int32_t ncols;
  float* feats;
  float* base;
  float* a;
  float* z;
  int32_t* col;
  double* ecol;
} bg_learned_samples;

/* Samples of `cols` bands of one Davidson state into entries at .. at + cols*rows - 1 and
 * columns col0 .. col0 + cols - 1: x the Ritz vectors, hx = H x, target e the ideal
 * corrections, kinetic t_g, lambda the Ritz values; all device pointers, rows x cols
 * column-major (interleaved complex when is_complex), on `stream` (cudaStream_t). */
int bg_learned_samples_build(bg_ctx* ctx, int64_t rows, int32_t cols, int32_t is_complex, const double* x,
                             const double* hx, const double* target, const double* kinetic,
                             const double* lambda, int32_t col0, int64_t at, const bg_learned_samples* out,
                             void* stream);
/* loss = (1/ncols) sum_j (1 - |sum_g p_g z_g|^2 / (sum_g p_g^2 a_g |e_j|^2)) with
 * p = base exp(clamp(m(feats), -3, 3)) under the BF16 parameters `net` (device), and its
 * gradient with respect to them into grad (device, BG_LEARNED_PARAMS floats).  work:
 * device, at least 6 ncols + 1 + (n + 1) / 2 doubles.  loss (host) may be NULL; when
 * given, the call waits for the stream. */
int bg_learned_loss_grad(bg_ctx* ctx, const bg_learned_samples* samples, const uint16_t* net, float* grad,
                         double* work, double* loss, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected at `step` >= 1) on the FP32
 * master parameters, with their BF16 rounding written to net (all device). */
int bg_learned_adam(bg_ctx* ctx, float* master, float* m1, float* m2, const float* grad, uint16_t* net,
                    int32_t step, float lr, void* stream);

/* ------------------------------------------------------------ no-allocation apply */
/* No counterpart in the reference.  The local and kinetic part of H x for one k point,
 * y = gather(FFT(V(r) IFFT(scatter x)))/N + T x, computed without allocating device
 * memory: for callers whose device memory belongs to another runtime's pool (a
 * framework caching allocator, a server arena) or that may not allocate after start-up,
 * since cudaMalloc/cudaFree can synchronise the device and stall other streams.  All
 * pointers are device memory the caller owns: fft_index (npw flat C-order grid indices,
 * Miller modulo the grid), v_grid (n0*n1*n2 real, C order), kinetic (npw, Ha), x and y
 * (npw x cols complex, interleaved, column-major).  Intermediates live in one 32 MiB
 * scratch array that the library keeps on every device it is loaded on until the
 * process exits; cols*n0*n1*n2 must not exceed 2,097,152 (BG_ESHAPE otherwise).  The
 * first call on a device loads the library's module there if CUDA's lazy loading has
 * not done so yet (which reserves the 32 MiB) and resolves the scratch array's device
 * address, so make it before any stream capture on that device.  The work runs on
 * `stream` (cudaStream_t, NULL for the legacy stream) and the call returns once it has
 * finished, reporting BG_ESHAPE if an fft_index entry lies outside [0, n0*n1*n2) (such
 * rows are skipped, never accessed) and BG_ENONFINITE for a non-finite x.  Every call
 * reuses the same scratch: calls whose work may overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller. */
int bg_local_apply_noalloc(const int32_t dims[3], int64_t npw, const int32_t* fft_index,
                           const double* v_grid, const double* kinetic, const double* x, double* y,
                           int64_t cols, void* stream);

/* ------------------------------------------------------------ operand builders */
/* Restatements of the reference setup (host, FP64) for callers without the
 * reference engine.  Lattice vectors are the ROWS of rows[9] (Bohr). */
int bg_setup_volume(const double rows[9], double* volume);
/* Plane waves with 1/2|k+G|^2 <= ecut (Ha), sorted by |G|^2 then Miller index
 * (crates/dft-basis/src/lib.rs:233-265).  Call with capacity 0 to get *npw. */
int bg_setup_basis(const double rows[9], double ecut_ha, const double kfrac[3], int64_t capacity,
                   int64_t* npw, int32_t* miller, double* kpg, double* kpg2);
/* Alias-free grid over the 4*ecut density sphere (crates/dft-basis/src/lib.rs:414-455). */
int bg_setup_grid(const double rows[9], double ecut_ha, int32_t dims[3], int32_t required[3]);
/* Gamma mirror maps (crates/dft-basis/src/half.rs:41-99): nh = (npw+1)/2 entries each. */
int bg_setup_half_sphere(const int32_t* miller, int64_t npw, int64_t* plus, int64_t* minus);

/* One pseudopotential species on a radial mesh (Bohr), local part and D in Ha. */
typedef struct {
  double z_valence;
  int32_t mesh;
  const double* r;
  const double* rab;
  const double* local;        /* V_loc(r), Ha (form factor only)                 */
  int32_t nbeta;
  const int32_t* l;           /* angular momentum per projector                 */
  const int32_t* beta_len;    /* samples per projector (prefix of the mesh)     */
  const double* const* beta;  /* r*beta(r) per projector                        */
  const double* dij;          /* nbeta x nbeta row-major, Ha                     */
  int32_t natoms;
  const double* positions;    /* 3*natoms Cartesian Bohr                         */
} bg_species;

int bg_setup_projector_count(int32_t nspecies, const bg_species* species, int32_t* nproj,
                             int32_t* natoms);
/* Projector table at the momenta k+G (kpg 3*npw, kpg2 npw) of one basis. */
int bg_setup_projectors(double volume, int64_t npw, const double* kpg, const double* kpg2,
                        int32_t nspecies, const bg_species* species, double* table,
                        int32_t* channels, double* couplings);
/* Ewald ion-ion energy (Ha) of natoms point charges (Cartesian Bohr positions, 3 per
 * ion) in a neutralising background, eta = sqrt(pi) / Omega^(1/3) (the reference's
 * default scheme, crates/dft-physics/src/ewald.rs:376-447). */
int bg_setup_ewald(const double rows[9], int32_t natoms, const double* positions, const double* charges,
                   double* energy);
/* V_loc(|G|) (Ha) of one species at n wave numbers (crates/dft-upf/src/radial.rs:246-305). */
int bg_setup_local_form_factor(const bg_species* species, double volume, int64_t n,
                               const double* g, double* out);
/* Atomic charge form factor rho_atom(|G|) / Omega at n wave numbers q >= 0 from a species'
 * PP_RHOATOM samples (4 pi r^2 rho(r)) on its radial mesh (r, rab; mesh points):
 * out[k] = integral of rho_atom(r) j0(q_k r) dr / volume, Simpson in the mesh index with
 * rab (crates/dft-upf/src/radial.rs:40-47), j0 = 1 at q = 0.  Replaces the rho channel
 * of the reference's atomic start fields (crates/dft-engine/src/refstart.rs:1166-1230,
 * the exact per-shell quadrature of the Gamma start).  BG_ENONFINITE for non-finite
 * samples. */
int bg_setup_atomic_charge(int64_t mesh, const double* r, const double* rab, const double* rho_atom,
                           double volume, int64_t n, const double* q, double* out);

#ifdef __cplusplus
}
#endif
#endif /* BAANDI_GPU_H */
