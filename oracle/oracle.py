"""Oracle (test infrastructure only): Python bindings of the C++ FP64 restatement
(hpsi_oracle.cpp) plus dense-matrix restatements used to pin it.

Only tests/, the smoke check and bench.py's cpu_baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

from . import setup_ref as S

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.oracle_local_complex.argtypes = [ctypes.c_int] * 3 + [ctypes.c_int64, _i64p, _f64p, _f64p, _f64p, _f64p,
                                                                ctypes.c_int, ctypes.c_int]
        L.oracle_local_gamma.argtypes = [ctypes.c_int] * 3 + [ctypes.c_int64, _i64p, ctypes.c_int64, _i64p, _i64p,
                                                              _f64p, _f64p, _f64p, _f64p, ctypes.c_int, ctypes.c_int]
        L.oracle_fft3d.argtypes = [ctypes.c_int] * 3 + [_f64p, ctypes.c_int]
        _lib = L
    return _lib


def _couple(nl, w):
    """D per atom on the projections w (nproj x m): out_i = sum_j D_ij w_j within each atom's
    channels (distributed_complex.rs:326-336; Gamma distributed_real_gamma.rs:1184-1195)."""
    out = np.empty_like(w)
    off, coff = 0, 0
    flat = np.concatenate([np.asarray(c, dtype=np.float64).reshape(-1) for c in nl.couplings])
    for cnt in nl.channels:
        d = flat[coff:coff + cnt * cnt].reshape(cnt, cnt)
        out[off:off + cnt] = d @ w[off:off + cnt]
        off += cnt
        coff += cnt * cnt
    return out


def apply_complex(dims, index, vgrid, kinetic, nl, x, threads=0):
    """H x for one k point; x (npw, m) complex128. vgrid: real grid, C order.  Local part and
    kinetic in the C++ restatement; P (D (P^H x)) as dense products (numpy BLAS)."""
    x = np.asfortranarray(x, dtype=np.complex128)
    npw, m = x.shape
    xin = np.ascontiguousarray(x.T).view(np.float64).reshape(-1)
    y = np.zeros(npw * m * 2)
    rc = lib().oracle_local_complex(int(dims[0]), int(dims[1]), int(dims[2]), npw,
                                    np.ascontiguousarray(index, dtype=np.int64),
                                    np.ascontiguousarray(vgrid, dtype=np.float64).reshape(-1),
                                    np.ascontiguousarray(kinetic, dtype=np.float64), xin, y, m, threads)
    if rc != 0:
        raise ValueError("oracle_local_complex: shape error")
    out = np.asfortranarray(y.view(np.complex128).reshape(m, npw).T)
    if nl is not None and nl.table.shape[1]:
        p = nl.table
        w = (p.T @ x.conj()).conj()                 # P^H x
        out += p @ _couple(nl, w)
    return out


def apply_gamma(dims, index, plus, minus, vgrid, kinetic_orc, proj_orc, nl, x, threads=0):
    """H x on real ORC rows; x (n, m) float64."""
    x = np.asarray(x, dtype=np.float64)
    n, m = x.shape
    xin = np.ascontiguousarray(x.T).reshape(-1)
    y = np.zeros(n * m)
    rc = lib().oracle_local_gamma(int(dims[0]), int(dims[1]), int(dims[2]), n,
                                  np.ascontiguousarray(index, dtype=np.int64), len(plus),
                                  np.ascontiguousarray(plus, dtype=np.int64),
                                  np.ascontiguousarray(minus, dtype=np.int64),
                                  np.ascontiguousarray(vgrid, dtype=np.float64).reshape(-1),
                                  np.ascontiguousarray(kinetic_orc, dtype=np.float64), xin, y, m, threads)
    if rc != 0:
        raise ValueError("oracle_local_gamma: shape error")
    out = np.asfortranarray(y.reshape(m, n).T)
    if proj_orc is not None and proj_orc.shape[1]:
        q = proj_orc.T @ x                          # P^T x
        out += proj_orc @ _couple(nl, q)
    return out


def fft3d(grid, sign):
    """sign +1: to_real (no scale); sign -1: to_reciprocal (1/N)."""
    a = np.ascontiguousarray(grid, dtype=np.complex128).copy()
    rc = lib().oracle_fft3d(a.shape[0], a.shape[1], a.shape[2], a.view(np.float64).reshape(-1), int(sign))
    if rc != 0:
        raise ValueError("oracle_fft3d")
    return a


# ---------------------------------------------------------------- dense restatements
def dense_local(basis, coeff: dict):
    """V(G - G') matrix from Fourier coefficients {miller: complex} (the reference's
    dense recipe, crates/dft-physics/tests/all/hamiltonian.rs:315-327)."""
    m = basis.miller.astype(np.int64)
    n = len(m)
    out = np.zeros((n, n), dtype=np.complex128)
    keys = {tuple(k): v for k, v in coeff.items()}
    diff = m[:, None, :] - m[None, :, :]
    for key, val in keys.items():
        mask = np.all(diff == np.array(key)[None, None, :], axis=2)
        out[mask] += val
    return out


def dense_hamiltonian(basis, coeff: dict, nl):
    """Dense H = V(G-G') + 1/2|k+G|^2 delta + P D P^H."""
    h = dense_local(basis, coeff)
    h[np.diag_indices_from(h)] += 0.5 * basis.kpg2
    if nl is not None and nl.table.shape[1]:
        d = S.coupling_matrix(nl)
        h += nl.table @ d @ nl.table.conj().T
    return h


def sampled_potential(dims, coeff: dict):
    """Real grid V(r) = Re sum_G c_G exp(2 pi i m.f) (hamiltonian.rs test helper :132-150)."""
    f = [np.arange(d) / d for d in dims]
    fi, fj, fk = np.meshgrid(f[0], f[1], f[2], indexing="ij")
    v = np.zeros(dims, dtype=np.complex128)
    for m, c in coeff.items():
        v += c * np.exp(1j * S.TAU * (m[0] * fi + m[1] * fj + m[2] * fk))
    return v.real.copy()
