"""Field step of an SCF map on the GPU: Hartree and LDA-PZ fields of a density.

`FieldGrid` holds one FFT box (bg_fields_*); `lda_hartree(density)` returns the
Hartree-plus-xc potential, the Hartree potential and the three energies of
crates/dft-engine/src/refscf/map.rs:41-198 (LDA-PZ, no core density): `hartree` =
dV/2 sum rho V_H, `xc` = dV sum |rho| eps_xc, `xc_integral` = dV sum rho v_xc (Ha).
Densities are C-order grids, numpy (synchronous) or CUDA float64 tensors (results on
the device).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .hamiltonian import Context, SolverError, default_context


@dataclass
class Fields:
    hxc: object
    vh: object
    hartree: float
    xc: float
    xc_integral: float


class FieldGrid:
    def __init__(self, rows, dims, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        self.dims = [int(d) for d in dims]
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).reshape(9))
        d = (ctypes.c_int32 * 3)(*self.dims)
        h = ctypes.c_void_p()
        self._check(self._lib.bg_fields_create(self.ctx.handle, r.ctypes.data_as(ctypes.c_void_p),
                                               ctypes.cast(d, ctypes.c_void_p), ctypes.byref(h)))
        self.handle = h

    def _check(self, rc):
        if rc != L.BG_OK:
            raise SolverError(rc, f"{L.CODE_NAMES.get(rc, rc)}: {L.last_error(self.ctx.handle)}")

    def volume(self) -> float:
        v = ctypes.c_double()
        self._check(self._lib.bg_fields_volume(self.handle, ctypes.byref(v)))
        return v.value

    def set_stream(self, stream_ptr: int):
        self._check(self._lib.bg_fields_set_stream(self.handle, ctypes.c_void_p(stream_ptr)))

    def lda_hartree(self, density, hxc=None, vh=None) -> Fields:
        n = int(np.prod(self.dims))
        e = np.zeros(3)
        if isinstance(density, np.ndarray):
            rho = np.ascontiguousarray(density, dtype=np.float64)
            if rho.size != n:
                raise SolverError(L.BG_ESHAPE, "density must be the full grid")
            hxc = np.empty(self.dims) if hxc is None else hxc
            vh = np.empty(self.dims) if vh is None else vh
            for a in (hxc, vh):
                if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != n:
                    raise SolverError(L.BG_ESHAPE, "outputs must be C-ordered float64 grids")
            ptrs = (rho.ctypes.data, hxc.ctypes.data, vh.ctypes.data)
            kind = L.BG_PTR_HOST
        else:
            import torch
            for a in (density, hxc, vh):
                if a is not None and (a.dtype != torch.float64 or not a.is_cuda or not a.is_contiguous()
                                      or a.numel() != n):
                    raise SolverError(L.BG_ESHAPE, "device grids are contiguous float64 CUDA tensors")
            hxc = torch.empty(self.dims, dtype=torch.float64, device=density.device) if hxc is None else hxc
            vh = torch.empty(self.dims, dtype=torch.float64, device=density.device) if vh is None else vh
            ptrs = (density.data_ptr(), hxc.data_ptr(), vh.data_ptr())
            kind = L.BG_PTR_DEVICE
        self._check(self._lib.bg_fields_lda_hartree(self.handle, *(ctypes.c_void_p(p) for p in ptrs),
                                                    e.ctypes.data_as(ctypes.c_void_p), kind))
        return Fields(hxc, vh, float(e[0]), float(e[1]), float(e[2]))

    # -- the mixer's coefficient space (density half-sphere)
    def set_sphere(self, flat_index):
        idx = np.ascontiguousarray(flat_index, dtype=np.int64)
        self._check(self._lib.bg_fields_set_sphere(self.handle, idx.size, idx.ctypes.data_as(ctypes.c_void_p)))
        self.nsphere = idx.size

    def sphere_forward(self, density, out=None):
        """FFT(density)/N on the half sphere (complex coefficients)."""
        if isinstance(density, np.ndarray):
            rho = np.ascontiguousarray(density, dtype=np.float64)
            out = np.empty(self.nsphere, np.complex128) if out is None else out
            kind, pr, po = L.BG_PTR_HOST, rho.ctypes.data, out.ctypes.data
        else:
            import torch
            out = torch.empty(self.nsphere, dtype=torch.complex128, device=density.device) if out is None else out
            kind, pr, po = L.BG_PTR_DEVICE, density.data_ptr(), out.data_ptr()
        self._check(self._lib.bg_fields_sphere_forward(self.handle, ctypes.c_void_p(pr), ctypes.c_void_p(po), kind))
        return out

    def sphere_inverse(self, coeffs, out=None):
        """2 Re(sum_half c e^{iGr}) - Re c_0 on the grid."""
        if isinstance(coeffs, np.ndarray):
            c = np.ascontiguousarray(coeffs, dtype=np.complex128)
            out = np.empty(self.dims) if out is None else out
            kind, pc, po = L.BG_PTR_HOST, c.ctypes.data, out.ctypes.data
        else:
            import torch
            out = torch.empty(self.dims, dtype=torch.float64, device=coeffs.device) if out is None else out
            kind, pc, po = L.BG_PTR_DEVICE, coeffs.data_ptr(), out.data_ptr()
        self._check(self._lib.bg_fields_sphere_inverse(self.handle, ctypes.c_void_p(pc), ctypes.c_void_p(po), kind))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self._lib.bg_fields_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
