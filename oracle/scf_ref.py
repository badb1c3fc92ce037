"""Oracle (test infrastructure only): the SCF map and outer loop of the reference
(crates/dft-engine/src/refscf/driver.rs:479, 589-660, 838-870; map.rs:200-384, 413-467;
density.rs:27-237; profile.rs:49-51) restated on the CPU over the oracle's apply
(oracle.py), Davidson (davidson_ref.py), fields and band density (fields_ref.py) and
mixer (broyden_ref.py), fixed or Fermi-Dirac occupations.  The caller supplies the operands it
shares with the GPU run (ionic potential, start blocks, Ewald energy); everything else
is built here from the oracle setup.  Only tests/ import this module.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import broyden_ref as B
from . import davidson_ref as D
from . import fields_ref as F
from . import oracle as OR
from . import setup_ref as S


def next_ethr_ry(previous, dr2_ry, electrons):
    return max(min(previous, 0.1 * dr2_ry / max(electrons, 1.0)), 1e-13)


def fermi_dirac(energies, weights, electrons, theta):
    """crates/dft-physics/src/occupations.rs:57-235 (one channel of capacity 2):
    bracket widening from theta, bisection to 1e-13 relative, TS from the entropy of
    each fraction."""
    e = np.stack(energies)
    w = np.asarray(weights)[:, None]

    def parts(mu):
        x = (e - mu) / theta
        a = np.abs(x)
        t = np.exp(-a)
        q = t / (1 + t)
        p = np.where(x >= 0, q, 1 / (1 + t))
        return p, np.log1p(t) + a * q

    count = lambda mu: float(np.sum(w * 2 * parts(mu)[0]))
    width = theta
    while True:
        lo, hi = e.min() - width, e.max() + width
        if count(lo) <= electrons <= count(hi):
            break
        width *= 2
    for _ in range(256):
        mu = 0.5 * lo + 0.5 * hi
        c = count(mu)
        if abs(c - electrons) <= 1e-13 * electrons:
            break
        if c < electrons:
            lo = mu
        else:
            hi = mu
    p, s = parts(mu)
    return [2 * row for row in p], theta * float(np.sum(w * 2 * s))


def half(m):
    return m[0] > 0 or (m[0] == 0 and (m[1] > 0 or (m[1] == 0 and m[2] >= 0)))


@dataclass
class Result:
    energy: float
    converged: bool
    iterations: int
    free_energy: float = float("nan")
    energies: list = field(default_factory=list)
    dr2: list = field(default_factory=list)
    eigenvalues: list = field(default_factory=list)


class _K:
    def __init__(self, cell, ecut, k, dims, species, gamma):
        self.b = S.basis_at_k(cell, ecut, k)
        self.nl = S.nonlocal_table(self.b, cell.volume, species)
        self.idx = S.fft_flat(S.g_to_fft(self.b, dims), dims)
        self.gamma = gamma
        diag = S.static_diagonal(0.5 * self.b.kpg2, self.nl)
        if gamma:
            self.plus, self.minus, _ = S.half_sphere(self.b)
            self.korc = S.orc_kinetic(self.plus, self.b.kpg2)
            self.porc = S.orc_projectors(self.plus, self.nl.table)
            d = np.empty(len(diag))
            d[0] = diag[0]
            i = np.arange(1, len(self.plus))
            d[2 * i - 1] = diag[self.plus[1:]]
            d[2 * i] = diag[self.plus[1:]]
            self.diag = d
        else:
            self.diag = diag

    def apply(self, dims, v):
        if self.gamma:
            return lambda x: OR.apply_gamma(dims, self.idx, self.plus, self.minus, v, self.korc, self.porc, self.nl, x)
        return lambda x: OR.apply_complex(dims, self.idx, v, 0.5 * self.b.kpg2, self.nl, x)

    def local_change(self, dims, dv):
        """x -> (dv(r) x) on the plane-wave rows: the kept-HX update of
        crates/dft-physics/src/distributed_complex.rs:388-420 (no kinetic, no projectors)."""
        if self.gamma:
            zk = np.zeros_like(self.korc)
            return lambda x: OR.apply_gamma(dims, self.idx, self.plus, self.minus, dv, zk, None, self.nl, x)
        zk = np.zeros_like(self.b.kpg2)
        return lambda x: OR.apply_complex(dims, self.idx, dv, zk, None, x)

    def coefficients(self, x):
        return F.expand_orc(x, self.plus, self.minus) if self.gamma else x


def run(rows, species, ecut_ha, dims, kpoints, gamma_real, bands, v_ion, starts, ewald, threshold_ha=5e-9,
        max_iterations=60, beta=0.7, history=8, davidson_max_iterations=20, smearing_ha=None, thomas_fermi=False,
        kept_hx=True, pool=None, start_density=None):
    """The SCF outer loop.  kept_hx: each map's Davidson starts from the previous map's
    H X brought to the new potential (crates/dft-engine/src/refscf/kept_hx.rs:98-160).
    pool: k points split over ranks (an object with `local` (range of owned k points),
    `gather_eigenvalues(list) -> every k point's list` and `sum_partials(array) -> sum over
    ranks`, as the reference's KPool: crates/dft-engine/src/refscf/k_pool.rs:76-330);
    `starts` then holds the owned k points' blocks only.  start_density: the start n(r) on
    the grid (setup_ref.atomic_density); None: uniform N_e / Omega (refstart.rs:704-757)."""
    cell = S.Cell(np.asarray(rows, dtype=np.float64))
    vol = cell.volume
    electrons = float(sum(s.pseudo.z * np.atleast_2d(s.positions).shape[0] for s in species))
    nocc = int(np.ceil(electrons / 2 - 1e-12))
    occ = np.array([2.0 if b < nocc else 0.0 for b in range(bands)])
    local = pool.local if pool is not None else range(len(kpoints))
    ks = [_K(cell, ecut_ha, kpoints[i][0], dims, species, gamma_real and tuple(kpoints[i][0]) == (0.0, 0.0, 0.0))
          for i in local]
    weights_all = [wk for _, wk in kpoints]
    weights = [weights_all[i] for i in local]
    dens = S.basis_at_k(cell, 4.0 * ecut_ha)
    keep = np.array([half(m) for m in dens.miller.tolist()])
    flat = S.fft_flat(S.g_to_fft(dens, dims), dims)[keep]
    g2 = dens.kpg2[keep]
    g0 = int(np.nonzero(flat == 0)[0][0])
    mixer = B.Broyden(g2, np.ones(len(g2), bool), vol, electrons, vol, beta=beta, history=history,
                      thomas_fermi=thomas_fermi)
    npts = int(np.prod(dims))

    def forward(rho):
        return (np.fft.fftn(rho) / npts).reshape(-1)[flat]

    def inverse(c):
        grid = np.zeros(npts, np.complex128)
        grid[flat] = c
        return 2.0 * (np.fft.ifftn(grid.reshape(dims)) * npts).real - c[g0].real

    n = np.full(dims, electrons / vol) if start_density is None else np.asarray(start_density, dtype=np.float64)
    x = forward(n)
    x[g0] = electrons / vol
    orbitals = [np.array(s) for s in starts]
    kept = None
    ethr, last_dr2 = 1e-2, np.inf
    res = Result(np.nan, False, 0)
    for it in range(1, max_iterations + 1):
        if it > 1:
            ethr = next_ethr_ry(1e-2 if it == 2 else ethr, last_dr2, electrons)
        redo = False
        while True:
            hxc, vh, eh, ex, vx = F.fields(rows, n)
            v = v_ion + hxc
            v0 = v.mean()
            rho = np.zeros(dims)
            band_sum = 0.0
            sols = []
            for kk, (k, wk) in enumerate(zip(ks, weights)):
                hx0 = None
                if kept is not None:
                    v_old, hxs = kept
                    hx0 = hxs[kk] + k.local_change(dims, v - v_old)(orbitals[kk])
                sols.append(D.solve(k.apply(dims, v), orbitals[kk], k.diag + v0,
                                    D.Options(bands, ethr / 2.0, nocc, first_step=(it == 1 and not redo),
                                              max_iterations=davidson_max_iterations), start_hx=hx0))
            kept = (v, [s.hx for s in sols]) if kept_hx else None
            ts = 0.0
            vals = [s.eigenvalues for s in sols]
            if pool is not None:
                vals = pool.gather_eigenvalues(vals)
            occs = [occ] * len(vals)
            if smearing_ha is not None:
                occs, ts = fermi_dirac(vals, weights_all, electrons, smearing_ha)
            occ_local = occs[local.start:local.stop] if pool is not None else occs
            for k, wk, sol, o in zip(ks, weights, sols, occ_local):
                rho += F.band_density_sum(dims, k.idx, k.coefficients(sol.eigenvectors), wk * o, vol)
            if pool is not None:
                rho = pool.sum_partials(rho)
            for wk, v, o in zip(weights_all, vals, occs):
                band_sum += float(np.dot(wk * o, v))
            energy = band_sum - eh + ex - vx + ewald
            y = forward(rho)
            y[g0] = electrons / vol
            fres = y - x
            dr2 = B.metric_dot(mixer.weights, fres, fres)
            orbitals = [s.eigenvectors for s in sols]
            res.energies.append(energy)
            res.dr2.append(dr2)
            if it == 1 and not redo and dr2 < ethr * max(electrons, 1.0):
                ethr = next_ethr_ry(ethr, dr2, electrons)
                redo = True
                continue
            break
        last_dr2 = dr2
        res.energy, res.iterations, res.free_energy = energy, it, energy - ts
        res.eigenvalues = vals
        if dr2 < 2.0 * threshold_ha:
            res.converged = True
            break
        nxt, _ = mixer.update(x, fres)
        n = inverse(nxt)
        x = nxt
    return res
