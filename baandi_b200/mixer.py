"""Host-side mirror of the reference density mixer over the C ABI (bg_mixer_*).

`Broyden(g2, smooth, volume, electrons, metric_volume, profile)` and
`update(x, f) -> (next, Diagnostics)` follow crates/dft-engine/src/refscf/broyden.rs
(Profile defaults: beta 0.7, history 8, plain screening); `gamma()`,
`reduced_residual()` and `metric(a, b)` expose the quantities the reference's tests
read.  Vectors are complex128 numpy arrays (synchronous) or CUDA complex128 tensors.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .hamiltonian import Context, SolverError, default_context


@dataclass
class Profile:
    beta: float = 0.7
    history: int = 8
    thomas_fermi: bool = False


@dataclass
class Diagnostics:
    iteration: int
    occupancy: int
    inserted_slot: int | None
    gamma_l2: float
    gamma_max: float
    condition: float | None


class Broyden:
    def __init__(self, g2, smooth, volume, electrons, metric_volume, profile: Profile | None = None,
                 ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        p = profile or Profile()
        g = np.ascontiguousarray(g2, dtype=np.float64)
        s = np.ascontiguousarray(np.asarray(smooth, dtype=bool).astype(np.int32))
        if g.shape != s.shape:
            raise SolverError(L.BG_EINVAL, "g2 and smooth differ in length")
        self.n = g.size
        prof = L.MixerProfile(p.beta, p.history, 1 if p.thomas_fermi else 0)
        h = ctypes.c_void_p()
        self._check(self._lib.bg_mixer_create(self.ctx.handle, ctypes.byref(prof), self.n,
                                              g.ctypes.data_as(ctypes.c_void_p), s.ctypes.data_as(ctypes.c_void_p),
                                              float(volume), float(electrons), float(metric_volume), ctypes.byref(h)))
        self.handle = h

    def _check(self, rc):
        if rc != L.BG_OK:
            raise SolverError(rc, f"{L.CODE_NAMES.get(rc, rc)}: {L.last_error(self.ctx.handle)}")

    def _vec(self, v):
        if isinstance(v, np.ndarray) or not hasattr(v, "data_ptr"):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.complex128).reshape(-1))
            if a.size != self.n:
                raise SolverError(L.BG_ESHAPE, "vector length")
            return a, a.ctypes.data, L.BG_PTR_HOST
        import torch
        if v.dtype != torch.complex128 or not v.is_cuda or not v.is_contiguous() or v.numel() != self.n:
            raise SolverError(L.BG_ESHAPE, "device vectors are contiguous complex128 CUDA tensors")
        return v, v.data_ptr(), L.BG_PTR_DEVICE

    def update(self, x, f, out=None):
        xa, px, kx = self._vec(x)
        fa, pf, kf = self._vec(f)
        if kx != kf:
            raise SolverError(L.BG_EINVAL, "x and f must both be host or both be device vectors")
        if out is None:
            if kx == L.BG_PTR_HOST:
                out = np.empty(self.n, np.complex128)
            else:
                import torch
                out = torch.empty_like(xa)
        _, pn, _ = self._vec(out)
        d = L.MixerDiagnostics()
        self._check(self._lib.bg_mixer_update(self.handle, ctypes.c_void_p(px), ctypes.c_void_p(pf),
                                              ctypes.c_void_p(pn), kx, ctypes.byref(d)))
        return out, Diagnostics(d.iteration, d.occupancy, None if d.inserted_slot < 0 else d.inserted_slot,
                                d.gamma_l2, d.gamma_max, d.condition if d.occupancy > 0 else None)

    def set_stream(self, stream_ptr: int):
        self._check(self._lib.bg_mixer_set_stream(self.handle, ctypes.c_void_p(stream_ptr)))

    def gamma(self) -> np.ndarray:
        g = np.zeros(25)
        c = ctypes.c_int32()
        self._check(self._lib.bg_mixer_gamma(self.handle, g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(c)))
        return g[: c.value].copy()

    def reduced_residual(self) -> np.ndarray:
        out = np.empty(self.n, np.complex128)
        self._check(self._lib.bg_mixer_reduced_residual(self.handle, out.ctypes.data_as(ctypes.c_void_p),
                                                        L.BG_PTR_HOST))
        return out

    def metric(self, a, b) -> float:
        aa, pa, ka = self._vec(a)
        bb, pb, kb = self._vec(b)
        r = ctypes.c_double()
        self._check(self._lib.bg_mixer_metric(self.handle, ctypes.c_void_p(pa), ctypes.c_void_p(pb),
                                              ctypes.byref(r), ka))
        return r.value

    def close(self):
        if getattr(self, "handle", None):
            self._lib.bg_mixer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
