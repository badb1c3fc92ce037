"""Host-side mirror of the reference's Hamiltonian operators over the C ABI.

`ComplexHamiltonian` stands in for DistributedComplexHamiltonian (reference:
crates/dft-physics/src/distributed_complex.rs:58-386) and `RealGammaHamiltonian` for
DistributedRealHamiltonian (crates/dft-physics/src/distributed_real_gamma.rs:120-1352),
both with one rank, so the method names, argument meaning and errors follow the
reference: `new_owned`, `set_owned_potential(values, epoch)` (epochs strictly
increasing), `apply_block(x, out)` (out completely overwritten, shape of x,
at most `capacity` columns), `global_len`, `local_rows`, `diagonal_static`,
`kinetic_diagonal`.  Blocks are numpy arrays (host; synchronous) or CUDA torch
tensors (device; enqueued on the operator stream).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .operands import NonlocalTable, PlaneWaves


STAGES = ("sticks_inverse", "planes", "sticks_forward", "project", "couple", "back")


class SolverError(RuntimeError):
    """Reference SolverError::InvalidParameter / Application (crates/dft-solvers/src/lib.rs:42-57)."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class Context:
    """One CUDA device (bg_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = L.load()
        opts = L.DeviceOpts(device)
        h = ctypes.c_void_p()
        rc = self._lib.bg_ctx_create(ctypes.byref(opts), ctypes.byref(h))
        if rc != L.BG_OK:
            raise L.BaandiError(rc, L.last_error(None))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            self._lib.bg_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _Operator:
    _gamma = False

    def __init__(self, pw: PlaneWaves, dims, nl: NonlocalTable | None, capacity: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        self.dims = [int(d) for d in dims]
        self.npw = pw.npw
        self._miller = np.ascontiguousarray(pw.miller, dtype=np.int32)
        self._kinetic = np.ascontiguousarray(0.5 * pw.kpg2, dtype=np.float64)
        desc = L.BasisDesc(self.npw, _p(self._miller), _p(self._kinetic), (ctypes.c_int32 * 3)(*self.dims),
                           1 if pw.gamma else 0)
        if nl is not None and nl.table.shape[1] > 0:
            self._table = np.ascontiguousarray(nl.table.T).view(np.float64)
            self._channels = np.ascontiguousarray(nl.channels, dtype=np.int32)
            self._couplings = np.ascontiguousarray(nl.couplings, dtype=np.float64)
            proj = L.Projectors(nl.table.shape[1], _p(self._table), len(self._channels), _p(self._channels),
                                _p(self._couplings))
            pproj = ctypes.byref(proj)
        else:
            pproj = None
        h = ctypes.c_void_p()
        create = self._lib.bg_op_create_gamma_real if self._gamma else self._lib.bg_op_create_complex
        rc = create(self.ctx.handle, ctypes.byref(desc), pproj, int(capacity), ctypes.byref(h))
        self._check(rc)
        self.handle = h
        self._capacity = int(capacity)
        self._epoch = None

    # -- reference accessors
    def global_len(self) -> int:
        return self.npw

    def local_rows(self):
        return np.arange(self.npw)

    def capacity(self) -> int:
        return self._capacity

    def owned_epoch(self):
        return self._epoch

    def diagonal_static(self) -> np.ndarray:
        out = np.zeros(self.npw)
        self._check(self._lib.bg_op_diagonal(self.handle, _p(out)))
        return out

    def _check(self, rc):
        if rc != L.BG_OK:
            raise SolverError(rc, f"{L.CODE_NAMES.get(rc, rc)}: {L.last_error(self.ctx.handle)}")

    def set_owned_potential(self, values, epoch: int):
        v = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1))
        if v.size != self.dims[0] * self.dims[1] * self.dims[2]:
            raise SolverError(L.BG_ESHAPE, "potential must be the full grid in C order")
        self._check(self._lib.bg_op_set_potential(self.handle, _p(v), int(epoch)))
        self._epoch = int(epoch)

    def set_owned_potential_device(self, values, epoch: int):
        """set_owned_potential from a CUDA float64 tensor holding the C-order grid
        (checked on the device; a non-finite grid keeps the old potential)."""
        self._grid_tensor(values, "potential")
        self._check(self._lib.bg_op_set_potential_ptr(self.handle, ctypes.c_void_p(values.data_ptr()), int(epoch),
                                                      L.BG_PTR_DEVICE))
        self._epoch = int(epoch)

    def _grid_points(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]

    def _grid_tensor(self, t, what):
        import torch
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.numel() != self._grid_points():
            raise SolverError(L.BG_ESHAPE, f"{what} must be a contiguous float64 CUDA tensor of the full grid")

    def _block_kind(self, x):
        """(pointer, columns, kind) of a block: numpy (npw, m) Fortran order or a CUDA
        tensor shaped (m, npw) row-major, the layouts of apply_block."""
        if isinstance(x, np.ndarray):
            want = np.float64 if self._gamma else np.complex128
            if x.ndim != 2 or x.shape[0] != self.npw or x.dtype != want or not x.flags.f_contiguous:
                raise SolverError(L.BG_ESHAPE, f"host blocks are Fortran-ordered {np.dtype(want).name} (npw, m)")
            return x.ctypes.data, x.shape[1], L.BG_PTR_HOST
        import torch
        want = torch.float64 if self._gamma else torch.complex128
        if x.dtype != want or not x.is_cuda or x.dim() != 2 or x.shape[1] != self.npw or not x.is_contiguous():
            raise SolverError(L.BG_ESHAPE, f"device blocks are contiguous {want} CUDA tensors shaped (m, npw)")
        return x.data_ptr(), x.shape[0], L.BG_PTR_DEVICE

    def add_local_change(self, x, change, hx):
        """hx += (change(r) x) on the plane-wave rows: the kept-HX update
        H_new x = H_old x + (V_new - V_old) x (reference add_local_change,
        crates/dft-physics/src/distributed_complex.rs:388-420).  x and hx are blocks in
        the layout of apply_block (both numpy or both CUDA tensors, hx updated in place);
        change is the C-order grid, numpy with numpy blocks, a CUDA float64 tensor with
        device blocks."""
        px, cols, kind = self._block_kind(x)
        ph, hcols, hkind = self._block_kind(hx)
        if hcols != cols or hkind != kind:
            raise SolverError(L.BG_ESHAPE, "hx must match x")
        if kind == L.BG_PTR_HOST:
            dv = np.ascontiguousarray(np.asarray(change, dtype=np.float64).reshape(-1))
            if dv.size != self._grid_points():
                raise SolverError(L.BG_ESHAPE, "change must be the full grid in C order")
            pc = dv.ctypes.data
        else:
            self._grid_tensor(change, "change")
            pc = change.data_ptr()
        self._check(self._lib.bg_op_add_local_change(self.handle, ctypes.c_void_p(px), ctypes.c_void_p(pc),
                                                     ctypes.c_void_p(ph), self.npw, int(cols), kind))
        return hx

    def band_density_sum(self, x, weights, volume: float, out=None, accumulate: bool = False):
        """sum_b weights[b] |psi_b(r)|^2 / volume on the C-order grid, bands in order
        (reference band_density_sum, distributed_complex.rs:485-547 and
        distributed_real_gamma.rs:744-785).  Numpy x gives a numpy (n0, n1, n2) grid;
        a CUDA x a CUDA float64 tensor.  accumulate adds into `out` (k-point sums)."""
        px, cols, kind = self._block_kind(x)
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
        if w.size != cols:
            raise SolverError(L.BG_ESHAPE, "one weight per column")
        if kind == L.BG_PTR_HOST:
            if out is None:
                out = np.zeros(self.dims)
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != self._grid_points():
                raise SolverError(L.BG_ESHAPE, "out must be a C-ordered float64 grid")
            pd = out.ctypes.data
        else:
            import torch
            if out is None:
                out = torch.zeros(self.dims, dtype=torch.float64, device=x.device)
            self._grid_tensor(out, "out")
            pd = out.data_ptr()
        self._check(self._lib.bg_op_band_density_sum(self.handle, ctypes.c_void_p(px), self.npw, int(cols), _p(w),
                                                     float(volume), ctypes.c_void_p(pd), 1 if accumulate else 0,
                                                     kind))
        return out

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self._lib.bg_op_stream(self.handle, ctypes.byref(s)))
        return s.value

    def set_stream(self, stream_ptr: int):
        self._check(self._lib.bg_op_set_stream(self.handle, ctypes.c_void_p(stream_ptr)))

    def sync(self):
        self._check(self._lib.bg_op_sync(self.handle))

    def launches(self) -> int:
        n = ctypes.c_int64()
        self._check(self._lib.bg_op_launches(self.handle, ctypes.byref(n)))
        return n.value

    def profile(self, enable: bool = True):
        """Record CUDA events around every stage of the following applies."""
        self._check(self._lib.bg_op_profile(self.handle, 1 if enable else 0))

    def stage_times(self) -> np.ndarray:
        """Milliseconds of the last apply's six stages (STAGES order)."""
        out = np.zeros(len(STAGES))
        self._check(self._lib.bg_op_stage_times(self.handle, _p(out)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self._lib.bg_op_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def is_real(self) -> bool:
        return self._gamma

    # -- apply
    precision = L.BG_PREC_FP64   # BG_PREC_FP32: the local part of apply_block in FP32

    def _apply_raw(self, x_ptr, y_ptr, cols, kind):
        self._check(self._lib.bg_op_apply_block(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                                self.npw, int(cols), kind, self.precision))


class ComplexHamiltonian(_Operator):
    """y = H x on complex plane-wave rows of one k point."""

    _gamma = False

    @classmethod
    def new_owned(cls, pw, dims, nl, capacity, ctx=None):
        return cls(pw, dims, nl, capacity, ctx)

    def kinetic_diagonal(self) -> np.ndarray:
        return self._kinetic.copy()

    def apply_block(self, x, out=None):
        """x: (npw, m) complex128 numpy array or CUDA complex128 torch tensor whose
        columns are contiguous (Fortran order / .T of a row-major (m, npw))."""
        if isinstance(x, np.ndarray):
            if x.ndim != 2 or x.shape[0] != self.npw:
                raise SolverError(L.BG_ESHAPE, "block rows")
            xin = np.asfortranarray(x, dtype=np.complex128)
            y = np.zeros_like(xin, order="F") if out is None else out
            if not (y.flags.f_contiguous and y.dtype == np.complex128 and y.shape == xin.shape):
                raise SolverError(L.BG_ESHAPE, "out must be a Fortran-ordered complex128 array of x's shape")
            self._apply_raw(xin.ctypes.data, y.ctypes.data, xin.shape[1], L.BG_PTR_HOST)
            return y
        return _apply_torch(self, x, out, complex_rows=True)


class RealGammaHamiltonian(_Operator):
    """y = H x on real ORC rows of the Gamma sphere (two columns per complex FFT)."""

    _gamma = True

    @classmethod
    def new_owned(cls, pw, dims, nl, capacity, ctx=None):
        if not pw.gamma:
            raise SolverError(L.BG_ESHAPE, "the real operator needs the Gamma sphere")
        return cls(pw, dims, nl, capacity, ctx)

    def kinetic_diagonal(self) -> np.ndarray:
        from .operands import half_sphere
        plus, _ = half_sphere(self._miller)
        out = np.empty(self.npw)
        out[0] = self._kinetic[0]
        i = np.arange(1, len(plus))
        out[2 * i - 1] = self._kinetic[plus[1:]]
        out[2 * i] = self._kinetic[plus[1:]]
        return out

    def apply_block(self, x, out=None):
        if isinstance(x, np.ndarray):
            if x.ndim != 2 or x.shape[0] != self.npw:
                raise SolverError(L.BG_ESHAPE, "block rows")
            xin = np.asfortranarray(x, dtype=np.float64)
            y = np.zeros_like(xin, order="F") if out is None else out
            if not (y.flags.f_contiguous and y.dtype == np.float64 and y.shape == xin.shape):
                raise SolverError(L.BG_ESHAPE, "out must be a Fortran-ordered float64 array of x's shape")
            self._apply_raw(xin.ctypes.data, y.ctypes.data, xin.shape[1], L.BG_PTR_HOST)
            return y
        return _apply_torch(self, x, out, complex_rows=False)


def _apply_torch(op, x, out, complex_rows):
    """Device path: x, out are CUDA tensors shaped (m, npw) row-major (one band per
    row, i.e. column-major (npw, m)); enqueued on the operator's stream."""
    import torch

    want = torch.complex128 if complex_rows else torch.float64
    if x.dtype != want or not x.is_cuda or x.dim() != 2 or x.shape[1] != op.npw or not x.is_contiguous():
        raise SolverError(L.BG_ESHAPE, f"device blocks are contiguous {want} CUDA tensors shaped (m, npw)")
    if out is None:
        out = torch.empty_like(x)
    if out.shape != x.shape or out.dtype != x.dtype or not out.is_contiguous():
        raise SolverError(L.BG_ESHAPE, "out must match x")
    op._apply_raw(x.data_ptr(), out.data_ptr(), x.shape[0], L.BG_PTR_DEVICE)
    return out


class KPointSet:
    """Several k-point operators of one grid applied in one batched launch per stage
    (bg_kset_*).  The reference applies them one after another
    (crates/dft-engine/src/refscf/k_map.rs:136-210); results are identical to the
    per-operator applies."""

    precision = L.BG_PREC_FP64   # BG_PREC_FP32: the local part of every apply in FP32

    def __init__(self, ops, ctx: Context | None = None):
        self.ctx = ctx or ops[0].ctx
        self._lib = self.ctx._lib
        self.ops = list(ops)
        arr = (ctypes.c_void_p * len(ops))(*[o.handle.value for o in ops])
        h = ctypes.c_void_p()
        rc = self._lib.bg_kset_create(self.ctx.handle, len(ops), ctypes.cast(arr, ctypes.c_void_p), ctypes.byref(h))
        if rc != L.BG_OK:
            raise SolverError(rc, f"{L.CODE_NAMES.get(rc, rc)}: {L.last_error(self.ctx.handle)}")
        self.handle = h

    def _check(self, rc):
        if rc != L.BG_OK:
            raise SolverError(rc, f"{L.CODE_NAMES.get(rc, rc)}: {L.last_error(self.ctx.handle)}")

    def apply_raw(self, x_ptrs, y_ptrs, cols, kind):
        n = len(self.ops)
        xa = (ctypes.c_void_p * n)(*x_ptrs)
        ya = (ctypes.c_void_p * n)(*y_ptrs)
        ca = (ctypes.c_int64 * n)(*[int(c) for c in cols])
        self._check(self._lib.bg_kset_apply(self.handle, ctypes.cast(xa, ctypes.c_void_p),
                                            ctypes.cast(ya, ctypes.c_void_p), ctypes.cast(ca, ctypes.c_void_p),
                                            kind, self.precision))

    def apply_blocks(self, xs, outs=None):
        """Host blocks (list of Fortran-ordered arrays, one per operator) -> list of H x."""
        if isinstance(xs[0], np.ndarray):
            xin = [np.asfortranarray(x) for x in xs]
            ys = outs if outs is not None else [np.zeros_like(x, order="F") for x in xin]
            self.apply_raw([x.ctypes.data for x in xin], [y.ctypes.data for y in ys], [x.shape[1] for x in xin],
                           L.BG_PTR_HOST)
            return ys
        import torch
        ys = outs if outs is not None else [torch.empty_like(x) for x in xs]
        self.apply_raw([x.data_ptr() for x in xs], [y.data_ptr() for y in ys], [x.shape[0] for x in xs],
                       L.BG_PTR_DEVICE)
        return ys

    def set_potential_device(self, values, epoch: int):
        """The potential of every operator from one CUDA float64 C-order grid
        (bg_kset_set_potential_ptr): checked and transposed once, copied to each
        operator on the set's stream."""
        self.ops[0]._grid_tensor(values, "potential")
        self._check(self._lib.bg_kset_set_potential_ptr(self.handle, ctypes.c_void_p(values.data_ptr()), int(epoch),
                                                        L.BG_PTR_DEVICE))
        for op in self.ops:
            op._epoch = int(epoch)

    def band_density_sum(self, xs, weights, volume: float, out=None, accumulate: bool = False):
        """sum over k of ops[k].band_density_sum(xs[k], weights[k], volume) in one batched
        launch per stage (bg_kset_band_density_sum): xs CUDA blocks shaped (m, npw_k),
        weights (n_k, m) on the host, out a CUDA float64 grid."""
        import torch
        n = len(self.ops)
        if len(xs) != n:
            raise SolverError(L.BG_ESHAPE, "one block per operator")
        cols = None
        for op, x in zip(self.ops, xs):
            px, c, kind = op._block_kind(x)
            if kind != L.BG_PTR_DEVICE:
                raise SolverError(L.BG_ESHAPE, "the set's band density takes CUDA blocks")
            if cols is not None and c != cols:
                raise SolverError(L.BG_ESHAPE, "every block has the same columns")
            cols = c
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(n, -1))
        if w.shape[1] != cols:
            raise SolverError(L.BG_ESHAPE, "one weight per column of each block")
        if out is None:
            out = torch.zeros(self.ops[0].dims, dtype=torch.float64, device=xs[0].device)
        self.ops[0]._grid_tensor(out, "out")
        xa = (ctypes.c_void_p * n)(*[x.data_ptr() for x in xs])
        self._check(self._lib.bg_kset_band_density_sum(self.handle, ctypes.cast(xa, ctypes.c_void_p), int(cols), _p(w),
                                                       float(volume), ctypes.c_void_p(out.data_ptr()),
                                                       1 if accumulate else 0, L.BG_PTR_DEVICE))
        return out

    def set_stream(self, stream_ptr: int):
        self._check(self._lib.bg_kset_set_stream(self.handle, ctypes.c_void_p(stream_ptr)))

    def sync(self):
        self._check(self._lib.bg_kset_sync(self.handle))

    def launches(self) -> int:
        n = ctypes.c_int64()
        self._check(self._lib.bg_kset_launches(self.handle, ctypes.byref(n)))
        return n.value

    def profile(self, enable: bool = True):
        self._check(self._lib.bg_kset_profile(self.handle, 1 if enable else 0))

    def stage_times(self) -> np.ndarray:
        out = np.zeros(len(STAGES))
        self._check(self._lib.bg_kset_stage_times(self.handle, _p(out)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self._lib.bg_kset_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DenseOperator(_Operator):
    """y = H x for an explicit rows x rows matrix (fixtures and exact small tests of the
    solver); real when H is real, complex otherwise."""

    def __init__(self, h: np.ndarray, capacity: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        h = np.asarray(h)
        self._gamma = not np.iscomplexobj(h)
        self._h = np.asfortranarray(h, dtype=np.float64 if self._gamma else np.complex128)
        self.npw = h.shape[0]
        self.dims = [0, 0, 0]
        hh = ctypes.c_void_p()
        self._check(self._lib.bg_op_create_dense(self.ctx.handle, self.npw, self._h.ctypes.data_as(ctypes.c_void_p),
                                                 0 if self._gamma else 1, int(capacity), ctypes.byref(hh)))
        self.handle = hh
        self._capacity = int(capacity)
        self._epoch = 0

    def apply_block(self, x, out=None):
        dt = np.float64 if self._gamma else np.complex128
        xin = np.asfortranarray(x, dtype=dt)
        y = np.zeros_like(xin, order="F") if out is None else out
        self._apply_raw(xin.ctypes.data, y.ctypes.data, xin.shape[1], L.BG_PTR_HOST)
        return y
