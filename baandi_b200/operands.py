"""Operand builders of the Hamiltonian apply, through the C ABI's bg_setup_* calls:
cell volume, plane-wave spheres, alias-free grids, Gamma mirror maps, projector
tables and local form factors (host, FP64).  These restate the reference's setup
(crates/dft-basis/src/lib.rs, crates/dft-physics/src/hamiltonian.rs:2605-2760,
crates/dft-upf/src/radial.rs) for callers without the reference engine.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _rows(rows):
    r = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).reshape(9))
    return r


def volume(rows) -> float:
    out = ctypes.c_double()
    r = _rows(rows)
    L.check(L.load().bg_setup_volume(_ptr(r), ctypes.byref(out)))
    return out.value


@dataclass
class PlaneWaves:
    """Sphere of one k point: Miller indices (npw, 3) sorted by |G|^2 then Miller,
    k+G (npw, 3) and |k+G|^2."""

    miller: np.ndarray
    kpg: np.ndarray
    kpg2: np.ndarray
    kfrac: tuple

    @property
    def npw(self):
        return len(self.miller)

    @property
    def gamma(self):
        return tuple(self.kfrac) == (0.0, 0.0, 0.0)


def wrap_fractional(k):
    """Fractional k canonicalised to [-1/2, 1/2) (crates/dft-geometry/src/kpoints.rs:21-32)."""
    return tuple(float(x) if -0.5 <= x < 0.5 else float(x - math.floor(x + 0.5)) for x in k)


def plane_waves(rows, ecut_ha: float, kfrac=(0.0, 0.0, 0.0)) -> PlaneWaves:
    lib = L.load()
    r = _rows(rows)
    k = np.ascontiguousarray(np.asarray(kfrac, dtype=np.float64))
    n = ctypes.c_int64()
    L.check(lib.bg_setup_basis(_ptr(r), ecut_ha, _ptr(k), 0, ctypes.byref(n), None, None, None))
    npw = n.value
    miller = np.zeros((npw, 3), np.int32)
    kpg = np.zeros((npw, 3))
    kpg2 = np.zeros(npw)
    L.check(lib.bg_setup_basis(_ptr(r), ecut_ha, _ptr(k), npw, ctypes.byref(n), _ptr(miller), _ptr(kpg), _ptr(kpg2)))
    return PlaneWaves(miller, kpg, kpg2, wrap_fractional(kfrac))


def grid(rows, ecut_ha: float):
    """(dims, required): the alias-free FFT grid over the 4*Ecut density sphere."""
    r = _rows(rows)
    d = np.zeros(3, np.int32)
    q = np.zeros(3, np.int32)
    L.check(L.load().bg_setup_grid(_ptr(r), ecut_ha, _ptr(d), _ptr(q)))
    return [int(x) for x in d], [int(x) for x in q]


def half_sphere(miller: np.ndarray):
    """Gamma mirror maps (plus, minus), crates/dft-basis/src/half.rs:41-99."""
    m = np.ascontiguousarray(miller, dtype=np.int32)
    nh = (len(m) + 1) // 2
    plus = np.zeros(nh, np.int64)
    minus = np.zeros(nh, np.int64)
    L.check(L.load().bg_setup_half_sphere(_ptr(m), len(m), _ptr(plus), _ptr(minus)))
    return plus, minus


def fft_index(miller: np.ndarray, dims, gamma: bool) -> np.ndarray:
    """Flat C-order grid index of every row (Miller modulo the grid)."""
    m = miller.astype(np.int64)
    idx = np.mod(m, np.asarray(dims, dtype=np.int64)[None, :])
    if gamma:
        for i in range(3):
            n = dims[i]
            if np.any(m[:, i] < -(n // 2)) or np.any(m[:, i] > (n - 1) // 2):
                raise ValueError("Miller index outside the canonical interval")
    return (idx[:, 0] * dims[1] + idx[:, 1]) * dims[2] + idx[:, 2]


@dataclass
class Pseudo:
    """Norm-conserving pseudopotential on a radial mesh (Bohr); local part and D in Ha;
    beta[i] holds r*beta_i(r) (the UPF PP_BETA convention)."""

    z: float
    r: np.ndarray
    rab: np.ndarray
    local: np.ndarray
    l: list
    beta: list
    dij: np.ndarray
    rho_atom: np.ndarray | None = None  # PP_RHOATOM: 4 pi r^2 rho_atom(r) on the mesh


@dataclass
class Species:
    pseudo: Pseudo
    positions: np.ndarray  # (natoms, 3) Cartesian Bohr
    _keep: list = field(default_factory=list, repr=False)

    def desc(self) -> L.SpeciesDesc:
        p = self.pseudo
        arrs = [np.ascontiguousarray(p.r, dtype=np.float64), np.ascontiguousarray(p.rab, dtype=np.float64),
                np.ascontiguousarray(p.local, dtype=np.float64)]
        ls = np.asarray(p.l, dtype=np.int32)
        lens = np.asarray([len(b) for b in p.beta], dtype=np.int32)
        betas = [np.ascontiguousarray(b, dtype=np.float64) for b in p.beta]
        bptr = (ctypes.c_void_p * max(1, len(betas)))(*[b.ctypes.data for b in betas])
        dij = np.ascontiguousarray(p.dij, dtype=np.float64).reshape(-1)
        pos = np.ascontiguousarray(np.atleast_2d(self.positions), dtype=np.float64).reshape(-1)
        self._keep = arrs + [ls, lens, dij, pos, bptr] + betas
        return L.SpeciesDesc(float(p.z), len(p.r), _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), len(betas),
                             _ptr(ls), _ptr(lens), ctypes.cast(bptr, ctypes.c_void_p), _ptr(dij),
                             int(np.atleast_2d(self.positions).shape[0]), _ptr(pos))


@dataclass
class NonlocalTable:
    """Projector columns (npw, nproj) complex, per-atom channel counts and D blocks."""

    table: np.ndarray
    channels: np.ndarray
    couplings: np.ndarray


def projectors(vol: float, pw: PlaneWaves, species) -> NonlocalTable:
    lib = L.load()
    descs = (L.SpeciesDesc * max(1, len(species)))(*[s.desc() for s in species])
    nproj = ctypes.c_int32()
    natoms = ctypes.c_int32()
    L.check(lib.bg_setup_projector_count(len(species), descs, ctypes.byref(nproj), ctypes.byref(natoms)))
    np_, na = nproj.value, natoms.value
    table = np.zeros((np_, pw.npw), np.complex128)  # column-major (npw x nproj) storage
    channels = np.zeros(max(1, na), np.int32)
    nd = sum(sum((2 * l + 1) for l in s.pseudo.l) ** 2 * np.atleast_2d(s.positions).shape[0] for s in species)
    couplings = np.zeros(max(1, nd))
    kpg = np.ascontiguousarray(pw.kpg)
    kpg2 = np.ascontiguousarray(pw.kpg2)
    L.check(lib.bg_setup_projectors(vol, pw.npw, _ptr(kpg), _ptr(kpg2), len(species), descs, _ptr(table),
                                    _ptr(channels), _ptr(couplings)))
    return NonlocalTable(table.T, channels[:na], couplings[:nd])


def ewald(rows, species) -> float:
    """Ion-ion Ewald energy (Ha) of the species' ions with charge Z_valence."""
    pos = np.ascontiguousarray(np.concatenate([np.atleast_2d(s.positions) for s in species]), dtype=np.float64)
    z = np.ascontiguousarray(np.concatenate([np.full(np.atleast_2d(s.positions).shape[0], s.pseudo.z)
                                             for s in species]), dtype=np.float64)
    out = ctypes.c_double()
    L.check(L.load().bg_setup_ewald(_ptr(_rows(rows)), len(z), _ptr(pos), _ptr(z), ctypes.byref(out)))
    return out.value


def local_form_factor(species: Species, vol: float, g: np.ndarray) -> np.ndarray:
    g = np.ascontiguousarray(np.asarray(g, dtype=np.float64).reshape(-1))
    out = np.zeros_like(g)
    d = species.desc()
    L.check(L.load().bg_setup_local_form_factor(ctypes.byref(d), vol, len(g), _ptr(g), _ptr(out)))
    return out


def log_mesh(points: int = 1201, end: float = 12.0, r0: float = 0.02):
    """Logarithmic radial mesh r_i = r0 expm1(i dx), rab = dx (r + r0) of the
    reference's synthetic fixtures (scripts/gen_synthetic_upf.py:22-24)."""
    dx = math.log1p(end / r0) / (points - 1)
    r = np.array([r0 * math.expm1(i * dx) for i in range(points)])
    return r, dx * (r + r0)


def gaussian_pseudo(z: float, rc: float, l=(0, 1), r_beta=(1.0, 1.0), dij_diag=(3.0, 1.5),
                    points: int = 1201, rho_radius: float | None = None) -> Pseudo:
    """Synthetic pseudopotential: local -Z erf(r/rc)/r and projectors r^l exp(-(r/r_beta)^2)
    with a diagonal D (Ha); with rho_radius R, the atomic charge rho(r) = Z exp(-(r/R)^2) /
    (pi^(3/2) R^3) as PP_RHOATOM, 4 Z / (sqrt(pi) R^3) r^2 exp(-(r/R)^2) (the atomic variant
    of the reference's synthetic fixtures, scripts/gen_synthetic_upf.py:64-65)."""
    r, rab = log_mesh(points)
    local = np.empty_like(r)
    local[0] = -2.0 * z / (rc * math.sqrt(math.pi))
    local[1:] = -z * np.array([math.erf(x / rc) for x in r[1:]]) / r[1:]
    beta = [r ** (ll + 1) * np.exp(-(r / rb) ** 2) for ll, rb in zip(l, r_beta)]
    n = len(l)
    dij = np.zeros(n * n)
    for i, d in enumerate(dij_diag):
        dij[i * n + i] = d
    rho = None
    if rho_radius is not None:
        rho = 4.0 * z / (math.sqrt(math.pi) * rho_radius ** 3) * r * r * np.exp(-(r / rho_radius) ** 2)
    return Pseudo(z, r, rab, local, list(l), beta, dij, rho)


def has_atomic_charge(p: Pseudo) -> bool:
    """PP_RHOATOM on the whole mesh and not all zero (crates/dft-engine/src/refstart.rs:56-59)."""
    return p.rho_atom is not None and len(p.rho_atom) == len(p.r) and bool(np.any(np.asarray(p.rho_atom) != 0.0))


def atomic_charge_transform(p: Pseudo, vol: float, q: np.ndarray) -> np.ndarray:
    """rho_atom(|G|) / Omega at the wave numbers q (bg_setup_atomic_charge)."""
    q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).reshape(-1))
    out = np.zeros_like(q)
    r = np.ascontiguousarray(p.r, dtype=np.float64)
    rab = np.ascontiguousarray(p.rab, dtype=np.float64)
    rho = np.ascontiguousarray(p.rho_atom, dtype=np.float64)
    L.check(L.load().bg_setup_atomic_charge(len(r), _ptr(r), _ptr(rab), _ptr(rho), vol, len(q), _ptr(q), _ptr(out)))
    return out


def atomic_density(rows, ecut_ha: float, dims, species) -> np.ndarray | None:
    """The atomic start density on the grid (C order), or None for the uniform start when any
    species carries no atomic charge (crates/dft-engine/src/refstart.rs:704-757): rho(G) =
    sum_s rho_s(|G|) S_s(G) / Omega over the 4 Ecut density sphere, n(r) = sum_G rho(G)
    e^{iGr}, negative values set to 0, scaled so that sum n Omega / N_points = N_e."""
    if not all(has_atomic_charge(s.pseudo) for s in species):
        return None
    vol = volume(rows)
    dens = plane_waves(rows, 4.0 * ecut_ha)
    q2u, inv = np.unique(dens.kpg2, return_inverse=True)
    rg = np.zeros(dens.npw, np.complex128)
    for s in species:
        ff = atomic_charge_transform(s.pseudo, vol, np.sqrt(q2u))[inv]
        sf = np.zeros(dens.npw, np.complex128)
        for tau in np.atleast_2d(s.positions):
            sf += np.exp(-1j * (dens.kpg @ tau))
        rg += ff * sf
    box = np.zeros(dims, np.complex128)
    idx = np.mod(dens.miller.astype(np.int64), np.asarray(dims)[None, :])
    box[idx[:, 0], idx[:, 1], idx[:, 2]] = rg
    n = np.maximum(np.ascontiguousarray((np.fft.ifftn(box) * box.size).real), 0.0)
    electrons = float(sum(s.pseudo.z * np.atleast_2d(s.positions).shape[0] for s in species))
    charge = float(n.sum()) * vol / n.size
    if not math.isfinite(charge) or charge <= 0.0:
        raise ValueError("invalid atomic charge")
    return n * (electrons / charge)
