"""Host-side mirror of the reference block Davidson over the C ABI (bg_davidson_solve).

Options/Solution mirror crates/dft-solvers/src/ref_davidson.rs:39-93: `bands`,
`threshold` (occupied Ritz-change threshold, Ha), `occupied`, `first_step`,
`capacity` (0 = 2 bands), `max_iterations` (default 20); the band threshold rule is
ref_davidson.rs:70-76.  The solver applies H and forms every subspace product on the
GPU; exhaustion of max_iterations returns an explicitly unconverged solution.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .hamiltonian import SolverError, _Operator


@dataclass
class Options:
    bands: int
    threshold: float
    occupied: int
    first_step: bool = False
    capacity: int = 0
    max_iterations: int = 20
    preconditioner: str = "smooth"   # "smooth" (reference Davidson), "tpa", "ritz_shift", "learned"
    # "fp64"; "fp32" (the local part of every H apply in FP32); "tensor" (solve_kset only:
    # the precision form, tensor-core applies, H Grams and rotations until every active
    # residual is below 1e-4, then the FP64 solve from those Ritz vectors)
    apply_precision: str = "fp64"

    def band_threshold(self, band: int) -> float:
        if self.first_step or band < self.occupied:
            return self.threshold
        return max(5.0 * self.threshold, 5e-6)


@dataclass
class Solution:
    eigenvalues: np.ndarray
    eigenvectors: np.ndarray
    converged: np.ndarray
    iterations: int
    reduced_solves: int
    h_calls: int
    h_columns: int
    repairs: int
    contractions: int
    dropped: int
    fallbacks: int = 0   # 1: the learned preconditioner gave way to TPA
    tensor_iterations: int = 0   # precision form: iterations before the FP64 handover
    hx: object = None            # H applied to the eigenvectors (solve_kset with want_hx)


def preconditioner_denominator(hamiltonian_diagonal_ha, eigenvalue_ha):
    """Smooth positive diagonal regulariser of ref_davidson.rs:418-422 (the device kernel
    uses the same formula)."""
    x = 2.0 * (np.asarray(hamiltonian_diagonal_ha, dtype=np.float64) - eigenvalue_ha)
    z = np.abs(x - 1.0)
    return 0.25 * (np.where(x >= 1.0, 2.0 * x, 2.0) + 1.0 / (np.hypot(z, 1.0) + z))


PRECISIONS = {"fp64": L.BG_PREC_FP64, "fp32": L.BG_PREC_FP32, "tensor": L.BG_PREC_TENSOR}
PRECONDITIONERS = {"smooth": L.BG_PRECOND_SMOOTH, "tpa": L.BG_PRECOND_TPA, "ritz_shift": L.BG_PRECOND_RITZ_SHIFT,
                   "learned": L.BG_PRECOND_LEARNED}


def _options(options: Options, flags: int = 0):
    if options.preconditioner not in PRECONDITIONERS:
        raise SolverError(L.BG_EINVAL, f"preconditioner {options.preconditioner!r}")
    if options.apply_precision not in PRECISIONS:
        raise SolverError(L.BG_EINVAL, f"apply precision {options.apply_precision!r}")
    return L.DavidsonOptions(options.bands, options.threshold, options.occupied, 1 if options.first_step else 0,
                             options.capacity, options.max_iterations, flags, PRECONDITIONERS[options.preconditioner],
                             PRECISIONS[options.apply_precision])


def solve(operator: _Operator, start: np.ndarray, hamiltonian_diagonal: np.ndarray, options: Options) -> Solution:
    """Lowest `options.bands` eigenpairs of `operator` from `start` (rows x bands).
    `hamiltonian_diagonal` is the H diagonal for the smooth and Ritz-shift corrections
    and the kinetic diagonal for TPA (the reference builds TPA on kinetic_diagonal,
    crates/dft-engine/src/oracle/scf.rs:2346-2350)."""
    lib = L.load()
    real = operator.is_real()
    dt = np.float64 if real else np.complex128
    x0 = np.asfortranarray(start, dtype=dt)
    rows, n = x0.shape
    if rows != operator.global_len() or n != options.bands:
        raise SolverError(L.BG_ESHAPE, "start must be rows x bands")
    diag = np.ascontiguousarray(hamiltonian_diagonal, dtype=np.float64)
    o = _options(options)
    vals = np.zeros(n)
    vecs = np.zeros((rows, n), dtype=dt, order="F")
    conv = np.zeros(n, np.int32)
    st = L.DavidsonStats()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib.bg_davidson_solve(operator.handle, p(x0), p(diag), ctypes.byref(o), p(vals), p(vecs), p(conv),
                               ctypes.byref(st))
    operator._check(rc)
    return Solution(vals, vecs, conv.astype(bool), st.iterations, st.reduced_solves, st.h_calls, st.h_columns,
                    st.repairs, st.contractions, st.dropped, st.fallbacks)


REDUCED_FLAGS = {"auto": 0, "wide": 2, "block": 4}


def reduced_eigh(s, h, ctx=None):
    """All eigenpairs of the Hermitian pencil H C = S C diag(w) (m x m, m <= 1536) by the
    many-block path of the batched Davidson's reduced problem (bg_reduced_eigh): Cholesky
    of S with the reference's pivot rule, A = L^-1 H L^-H, Householder tridiagonalisation,
    bisection and inverse iteration, C = L^-H Y.  Returns (w ascending, C, device ms)."""
    from .hamiltonian import default_context
    ctx = ctx or default_context()
    h = np.asarray(h)
    complex_ = np.iscomplexobj(h) or np.iscomplexobj(s)
    dt = np.complex128 if complex_ else np.float64
    hm = np.asfortranarray(h, dtype=dt)
    sm = np.asfortranarray(s, dtype=dt)
    m = hm.shape[0]
    if hm.shape != (m, m) or sm.shape != (m, m):
        raise SolverError(L.BG_ESHAPE, "square pencil expected")
    w = np.zeros(m)
    c = np.zeros((m, m), dtype=dt, order="F")
    ms = ctypes.c_double()
    rc = L.load().bg_reduced_eigh(ctx.handle, m, 1 if complex_ else 0, sm.ctypes.data,
                                  hm.ctypes.data, w.ctypes.data, c.ctypes.data, ctypes.byref(ms))
    if rc != L.BG_OK:
        raise SolverError(rc, f"{L.CODE_NAMES.get(rc, rc)}: {L.last_error(ctx.handle)}")
    return w, c, ms.value


def solve_kset(kset, starts, diagonals, options: Options, graph: bool = True, reduced: str = "auto",
               start_hx=None, want_hx: bool = False):
    """The reference Davidson for every k point of a KPointSet at once
    (bg_kset_davidson_solve): each large product is one launch over all k points, the
    reduced problems and control decisions run on the GPU, and an iteration is one
    replayed CUDA graph (graph=False launches the same kernels one by one; reduced "wide"
    or "block" forces the many-block or the one-block reduced problem).  Device blocks
    only: start_hx (one block per k point, H applied to the start block, e.g. kept from the
    previous solve and updated with add_local_change) spares the start apply, and want_hx
    returns H X of the eigenvectors in Solution.hx (bg_kset_davidson_solve_hx).  starts /
    diagonals: one (rows_k x bands) block and one rows_k diagonal per k point, numpy
    (host) or CUDA tensors (device; blocks shaped (bands, rows_k) row-major, the layout
    of apply_block).  Returns one Solution per k point, eigenvectors on the same side."""
    lib = L.load()
    real = kset.ops[0].is_real()
    nk = len(kset.ops)
    if len(starts) != nk or len(diagonals) != nk:
        raise SolverError(L.BG_ESHAPE, "one start block and one diagonal per k point")
    n = options.bands
    device = not isinstance(starts[0], np.ndarray)
    if device:
        import torch
        want = torch.float64 if real else torch.complex128
        x0, dg = list(starts), list(diagonals)
        for op, x, d in zip(kset.ops, x0, dg):
            if (x.dtype != want or not x.is_cuda or not x.is_contiguous() or tuple(x.shape) != (n, op.global_len())
                    or d.dtype != torch.float64 or not d.is_cuda or d.numel() != op.global_len()):
                raise SolverError(L.BG_ESHAPE, "device starts are contiguous (bands, rows) CUDA tensors")
        vecs = [torch.empty_like(x) for x in x0]
        ptr = lambda a: a.data_ptr()
        kind = L.BG_PTR_DEVICE
    else:
        dt = np.float64 if real else np.complex128
        x0 = [np.asfortranarray(x, dtype=dt) for x in starts]
        dg = [np.ascontiguousarray(d, dtype=np.float64) for d in diagonals]
        for op, x, d in zip(kset.ops, x0, dg):
            if x.shape != (op.global_len(), n) or d.shape != (op.global_len(),):
                raise SolverError(L.BG_ESHAPE, "start must be rows x bands, diagonal rows")
        vecs = [np.zeros((op.global_len(), n), dtype=dt, order="F") for op in kset.ops]
        ptr = lambda a: a.ctypes.data
        kind = L.BG_PTR_HOST
    vals = [np.zeros(n) for _ in range(nk)]
    conv = [np.zeros(n, np.int32) for _ in range(nk)]
    stats = (L.DavidsonStats * nk)()
    o = _options(options, (0 if graph else 1) | REDUCED_FLAGS[reduced])
    arr = lambda lst, f: (ctypes.c_void_p * nk)(*[f(a) for a in lst])
    host = lambda a: a.ctypes.data
    hxs = None
    if start_hx is not None or want_hx:
        if not device:
            raise SolverError(L.BG_EINVAL, "kept H X blocks are device blocks")
        if start_hx is not None:
            start_hx = list(start_hx)
            if len(start_hx) != nk or any(h.dtype != x.dtype or not h.is_cuda or not h.is_contiguous()
                                          or h.shape != x.shape for h, x in zip(start_hx, x0)):
                raise SolverError(L.BG_ESHAPE, "start_hx: one contiguous block shaped like its start per k point")
        hxs = [torch.empty_like(x) for x in x0] if want_hx else None
        rc = lib.bg_kset_davidson_solve_hx(kset.handle, arr(x0, ptr), arr(start_hx, ptr) if start_hx else None,
                                           arr(dg, ptr), ctypes.byref(o), arr(vals, host), arr(vecs, ptr),
                                           arr(hxs, ptr) if hxs else None, arr(conv, host), stats)
    else:
        rc = lib.bg_kset_davidson_solve(kset.handle, arr(x0, ptr), arr(dg, ptr), ctypes.byref(o), kind,
                                        arr(vals, host), arr(vecs, ptr), arr(conv, host), stats)
    kset._check(rc)
    return [Solution(vals[k], vecs[k], conv[k].astype(bool), stats[k].iterations, stats[k].reduced_solves,
                     stats[k].h_calls, stats[k].h_columns, stats[k].repairs, stats[k].contractions, stats[k].dropped,
                     stats[k].fallbacks, stats[k].tensor_iterations, hxs[k] if hxs else None)
            for k in range(nk)]
