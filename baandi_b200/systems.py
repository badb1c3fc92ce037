"""Synthetic workloads of the Hamiltonian apply: the five silicon/aluminium cells the
benchmarks are quoted on, with seeded displacements, synthetic pseudopotentials,
k meshes and the ionic local potential V_ion(r) on the FFT grid.

All inputs are synthetic (no pseudopotential files or datasets): Gaussian-erf local
parts and r^l exp(-r^2) projectors on the reference's synthetic log mesh.  Seeds:
numpy default_rng(2026 + workload number).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import operands as O

SI_A = 10.26
DIAMOND_FRAC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                         [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
FCC_FRAC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])


def monkhorst_pack(grid, shift=(0.0, 0.0, 0.0)):
    """Uniform mesh (m + s)/n wrapped to [-1/2, 1/2), weights 1/count
    (crates/dft-geometry/src/kpoints.rs:63-88)."""
    count = grid[0] * grid[1] * grid[2]
    return [(O.wrap_fractional([(m + s) / n for m, s, n in zip((i, j, k), shift, grid)]), 1.0 / count)
            for i in range(grid[0]) for j in range(grid[1]) for k in range(grid[2])]


def reduce_time_reversal(points):
    """Merge k and -k modulo integers, keep the first (kpoints.rs:93-116)."""
    out = []
    for k, w in points:
        k = O.wrap_fractional(k)
        hit = None
        for p in out:
            for s in (1.0, -1.0):
                if all(abs((k[a] - s * p[0][a]) - round(k[a] - s * p[0][a])) <= 1e-12 for a in range(3)):
                    hit = p
                    break
            if hit:
                break
        if hit:
            hit[1] += w
        else:
            out.append([k, w])
    return [(tuple(k), w) for k, w in out]


@dataclass
class Workload:
    name: str
    rows: np.ndarray                  # lattice vectors as rows (Bohr)
    species: list                     # operands.Species
    ecut_ha: float
    bands: int
    occupied: int
    kpoints: list                     # [(kfrac, weight)]
    gamma_real: bool
    dims_override: list | None = None
    seed: int = 2026
    _dims: list | None = field(default=None, repr=False)

    @property
    def volume(self) -> float:
        return O.volume(self.rows)

    @property
    def natoms(self) -> int:
        return sum(np.atleast_2d(s.positions).shape[0] for s in self.species)

    def dims(self):
        if self._dims is None:
            d, req = O.grid(self.rows, self.ecut_ha)
            if self.dims_override is not None:
                if any(o < r for o, r in zip(self.dims_override, req)):
                    raise ValueError(f"override {self.dims_override} below required {req}")
                d = list(self.dims_override)
            self._dims = d
        return self._dims

    def plane_waves(self, k=(0.0, 0.0, 0.0)):
        return O.plane_waves(self.rows, self.ecut_ha, k)

    def nonlocal_table(self, pw):
        return O.projectors(self.volume, pw, self.species)

    def ionic_potential(self) -> np.ndarray:
        """V_ion(r) on the grid (C order): sum_species V_loc(|G|) S(G) over the
        4*Ecut density sphere, transformed with f(r) = sum_G f(G) e^{iGr}."""
        dims = self.dims()
        dens = O.plane_waves(self.rows, 4.0 * self.ecut_ha)
        vg = np.zeros(dens.npw, np.complex128)
        q2u, inv = np.unique(dens.kpg2, return_inverse=True)
        vol = self.volume
        for s in self.species:
            ff = O.local_form_factor(s, vol, np.sqrt(q2u))[inv]
            sf = np.zeros(dens.npw, np.complex128)
            # the atoms' phase factors on the host threads (numpy releases the GIL), added in
            # atom order: the same sum as one atom after another
            taus = np.atleast_2d(s.positions)
            for lo in range(0, len(taus), _PHASE_BATCH):
                for term in _map_threads(lambda tau: np.exp(-1j * (dens.kpg @ tau)), taus[lo:lo + _PHASE_BATCH]):
                    sf += term
            vg += ff * sf
        box = np.zeros(dims, np.complex128)
        idx = np.mod(dens.miller.astype(np.int64), np.asarray(dims)[None, :])
        box[idx[:, 0], idx[:, 1], idx[:, 2]] = vg
        v = np.fft.ifftn(box) * box.size
        return np.ascontiguousarray(v.real)

    def start_density(self) -> np.ndarray | None:
        """The atomic start density on the grid, or None (uniform) when a species has no
        atomic charge."""
        return O.atomic_density(self.rows, self.ecut_ha, self.dims(), self.species)

    def random_block(self, npw, cols, seed_offset=0, real=False):
        """Seeded random-phase columns c_G = e^{i theta}/sqrt(Npw) (real: ORC rows of unit norm)."""
        rng = np.random.default_rng(self.seed + seed_offset)
        if real:
            x = rng.standard_normal((npw, cols))
            return np.asfortranarray(x / np.linalg.norm(x, axis=0, keepdims=True))
        th = rng.uniform(0.0, 2.0 * math.pi, size=(npw, cols))
        out = np.empty((npw, cols), np.complex128, order="F")
        scale = math.sqrt(npw)

        def block(c0):
            out[:, c0:c0 + 32] = np.exp(1j * th[:, c0:c0 + 32]) / scale
        list(_map_threads(block, range(0, cols, 32)))
        return out


_PHASE_BATCH = 32


def _map_threads(fn, items):
    """fn over items on a pool of host threads, results in item order."""
    from concurrent.futures import ThreadPoolExecutor
    items = list(items)
    if len(items) <= 1:
        return [fn(x) for x in items]
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1, len(items))) as ex:
        return list(ex.map(fn, items))


def _si_pseudo(rho_radius=None):
    return O.gaussian_pseudo(4.0, 0.45, l=(0, 1), r_beta=(1.0, 1.0), dij_diag=(3.0, 1.5), rho_radius=rho_radius)


def _al_pseudo():
    return O.gaussian_pseudo(3.0, 0.55, l=(0, 1), r_beta=(1.0, 1.0), dij_diag=(3.0, 1.5))


def _supercell(frac, reps, a_cell, amp, rng):
    pts = []
    for i in range(reps):
        for j in range(reps):
            for k in range(reps):
                for f in frac:
                    pts.append((np.asarray(f) + [i, j, k]) / reps)
    pos = np.asarray(pts) * a_cell
    if amp > 0:
        pos = pos + rng.uniform(-amp, amp, size=pos.shape)
    return pos


def si2_gamma() -> Workload:
    """Si2 fcc primitive (a = 10.26 Bohr), Gamma real path, 30 Ry, 8 bands."""
    a = SI_A
    rows = np.array([[0, a / 2, a / 2], [a / 2, 0, a / 2], [a / 2, a / 2, 0]])
    pos = np.array([[0, 0, 0], [a / 4, a / 4, a / 4]])
    return Workload("si2_gamma_real_30ry", rows, [O.Species(_si_pseudo(), pos)], 15.0, 8, 4,
                    [((0.0, 0.0, 0.0), 1.0)], True, seed=2027)


def si2_gamma_atomic(radius: float = 1.0) -> Workload:
    """Si2 Gamma with a Gaussian atomic charge of `radius` Bohr: the atomic-density start."""
    w = si2_gamma()
    w.name = "si2_gamma_real_30ry_atomic"
    w.species = [O.Species(_si_pseudo(rho_radius=radius), s.positions) for s in w.species]
    return w


def si8_k444() -> Workload:
    """Si8 conventional cube (a = 10.26), 4x4x4 mesh reduced by time reversal to 36 k, 40 Ry, 24 bands."""
    a = SI_A
    rows = np.diag([a, a, a])
    pos = DIAMOND_FRAC * a
    ks = reduce_time_reversal(monkhorst_pack((4, 4, 4)))
    return Workload("si8_k444_40ry", rows, [O.Species(_si_pseudo(), pos)], 20.0, 24, 16, ks, False, seed=2028)


def si64_gamma() -> Workload:
    """Si64 2x2x2 cube (a = 20.52), +-0.05 Bohr seeded noise, Gamma complex path, 30 Ry, 160 bands."""
    rng = np.random.default_rng(2029)
    a = 2 * SI_A
    pos = _supercell(DIAMOND_FRAC, 2, a, 0.05, rng)
    return Workload("si64_gamma_30ry", np.diag([a, a, a]), [O.Species(_si_pseudo(), pos)], 15.0, 160, 128,
                    [((0.0, 0.0, 0.0), 1.0)], False, seed=2029)


def al32_k222(geometry_seed: int = 2030) -> Workload:
    """Al32 fcc 2x2x2 conventional (a = 15.30), +-0.08 seeded noise, 2x2x2 mesh (8 k), 30 Ry, grid 60^3, 64 bands.
    geometry_seed: the seed of the displacements and start blocks (2030: the benchmark cell)."""
    rng = np.random.default_rng(geometry_seed)
    a = 15.30
    pos = _supercell(FCC_FRAC, 2, a, 0.08, rng)
    ks = reduce_time_reversal(monkhorst_pack((2, 2, 2)))
    return Workload("al32_k222_30ry", np.diag([a, a, a]), [O.Species(_al_pseudo(), pos)], 15.0, 64, 48, ks, False,
                    dims_override=[60, 60, 60], seed=geometry_seed)


def si216_gamma() -> Workload:
    """Si216 3x3x3 cube (a = 30.78), +-0.05 seeded noise, Gamma complex path, 30 Ry, 480 bands."""
    rng = np.random.default_rng(2031)
    a = 3 * SI_A
    pos = _supercell(DIAMOND_FRAC, 3, a, 0.05, rng)
    return Workload("si216_gamma_30ry", np.diag([a, a, a]), [O.Species(_si_pseudo(), pos)], 15.0, 480, 432,
                    [((0.0, 0.0, 0.0), 1.0)], False, seed=2031)


WORKLOADS = {
    "si2": si2_gamma, "si2_atomic": si2_gamma_atomic, "si8": si8_k444, "si64": si64_gamma, "al32": al32_k222, "si216": si216_gamma,
}
