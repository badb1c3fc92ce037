"""Oracle (test infrastructure only): the five benchmark cells restated from the oracle's
own setup (setup_ref.py), so that the CPU baseline and bench.py's reference arm build
their operands without the product library.

Cells (lattice, seeded displacements, synthetic pseudopotentials, k meshes, cutoffs,
band counts) are those of the benchmark configurations; seeds are numpy
default_rng(2026 + workload number) for displacements and start blocks.  The grid
follows the reference's rule (crates/dft-basis/src/lib.rs:414-455) with the Al32
override of 60^3; V_ion(r) is the reference's ionic local potential
(crates/dft-physics/src/hamiltonian.rs:211-300) on the 4 Ecut density sphere, brought to
the grid with f(r) = sum_G f(G) e^{iGr}.

Only tests/ and bench.py (cpu_baseline leg, reference arm) import this module.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import setup_ref as S

SI_A = 10.26
DIAMOND_FRAC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                         [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
FCC_FRAC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])


@dataclass
class Cell:
    name: str
    rows: np.ndarray
    z: float
    rc: float
    positions: np.ndarray
    ecut_ha: float
    bands: int
    kpoints: list
    gamma_real: bool
    override: list | None = None
    seed: int = 2026
    rho_radius: float | None = None  # Gaussian atomic charge (PP_RHOATOM) of this radius
    _cache: dict = field(default_factory=dict, repr=False)

    @property
    def cell(self) -> S.Cell:
        return S.Cell(self.rows)

    @property
    def natoms(self) -> int:
        return len(self.positions)

    def species(self):
        ps = S.synthetic_pseudo(self.z, self.rc, (0, 1), (1.0, 1.0), np.diag([3.0, 1.5]).reshape(-1),
                                rho_radius=self.rho_radius)
        return [S.Species(ps, self.positions)]

    def dims(self):
        if "dims" not in self._cache:
            d, _ = S.grid_dims(self.cell, self.ecut_ha, self.override)
            self._cache["dims"] = list(d)
        return self._cache["dims"]

    def basis(self, k=(0.0, 0.0, 0.0)) -> S.Basis:
        return S.basis_at_k(self.cell, self.ecut_ha, k)

    def nonlocal_table(self, basis: S.Basis) -> S.Nonlocal:
        return S.nonlocal_table(basis, self.cell.volume, self.species())

    def fft_index(self, basis: S.Basis):
        dims = self.dims()
        return S.fft_flat(S.g_to_fft(basis, dims), dims)

    def ionic_potential(self) -> np.ndarray:
        """V_ion(r) on the grid (C order, real)."""
        if "v" not in self._cache:
            dims = self.dims()
            dens = S.basis_at_k(self.cell, 4.0 * self.ecut_ha)
            # S.ionic_local, with the form factor evaluated once per distinct |G|
            q2u, inv = np.unique(dens.gnorm2, return_inverse=True)
            vg = np.zeros(dens.npw, np.complex128)
            for sp in self.species():
                ff = S.local_form_factor(sp.pseudo, self.cell.volume, np.sqrt(q2u))[inv]
                sf = np.zeros(dens.npw, np.complex128)
                for tau in np.atleast_2d(sp.positions):
                    ang = (dens.gcart[:, 0] * tau[0] + dens.gcart[:, 1] * tau[1]) + dens.gcart[:, 2] * tau[2]
                    sf += np.cos(-ang) + 1j * np.sin(-ang)
                vg += ff * sf
            box = np.zeros(dims, np.complex128)
            idx = S.g_to_fft(dens, dims)
            box[idx[:, 0], idx[:, 1], idx[:, 2]] = vg
            v = np.fft.ifftn(box) * box.size
            self._cache["v"] = np.ascontiguousarray(v.real)
        return self._cache["v"]

    def random_block(self, npw, cols, seed_offset=0):
        """Seeded random-phase columns c_G = e^{i theta}/sqrt(Npw)."""
        rng = np.random.default_rng(self.seed + seed_offset)
        th = rng.uniform(0.0, 2.0 * math.pi, size=(npw, cols))
        return np.asfortranarray(np.exp(1j * th) / math.sqrt(npw))


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


def si2() -> Cell:
    a = SI_A
    rows = np.array([[0, a / 2, a / 2], [a / 2, 0, a / 2], [a / 2, a / 2, 0]])
    pos = np.array([[0, 0, 0], [a / 4, a / 4, a / 4]])
    return Cell("si2_gamma_real_30ry", rows, 4.0, 0.45, pos, 15.0, 8, [((0.0, 0.0, 0.0), 1.0)], True, seed=2027)


def si2_atomic(radius: float = 1.0) -> Cell:
    """Si2 with a Gaussian atomic charge of `radius` Bohr, the atomic-density start."""
    c = si2()
    c.rho_radius = radius
    return c


def si8() -> Cell:
    a = SI_A
    ks = S.reduce_time_reversal(S.monkhorst_pack((4, 4, 4)))
    return Cell("si8_k444_40ry", np.diag([a, a, a]), 4.0, 0.45, DIAMOND_FRAC * a, 20.0, 24, ks, False, seed=2028)


def si64() -> Cell:
    rng = np.random.default_rng(2029)
    a = 2 * SI_A
    pos = _supercell(DIAMOND_FRAC, 2, a, 0.05, rng)
    return Cell("si64_gamma_30ry", np.diag([a, a, a]), 4.0, 0.45, pos, 15.0, 160, [((0.0, 0.0, 0.0), 1.0)], False,
                seed=2029)


def al32() -> Cell:
    rng = np.random.default_rng(2030)
    a = 15.30
    pos = _supercell(FCC_FRAC, 2, a, 0.08, rng)
    ks = S.reduce_time_reversal(S.monkhorst_pack((2, 2, 2)))
    return Cell("al32_k222_30ry", np.diag([a, a, a]), 3.0, 0.55, pos, 15.0, 64, ks, False, override=[60, 60, 60],
                seed=2030)


def si216() -> Cell:
    rng = np.random.default_rng(2031)
    a = 3 * SI_A
    pos = _supercell(DIAMOND_FRAC, 3, a, 0.05, rng)
    return Cell("si216_gamma_30ry", np.diag([a, a, a]), 4.0, 0.45, pos, 15.0, 480, [((0.0, 0.0, 0.0), 1.0)], False,
                seed=2031)


CELLS = {"si2": si2, "si8": si8, "si64": si64, "al32": al32, "si216": si216}
