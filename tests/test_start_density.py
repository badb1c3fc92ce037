"""The atomic start density (crates/dft-engine/src/refstart.rs:704-757, the rho channel of
atomic_fields :1166-1230): the library's form factor (bg_setup_atomic_charge) against the
Gaussian's closed form, its grid density against the oracle's restatement, the reference's
rule for falling back to the uniform start, argument checks, and the oracle SCF from the
atomic start (CPU only)."""
import math

import numpy as np
import pytest

from baandi_b200 import _lib as L
from baandi_b200 import operands as O
from baandi_b200 import systems as W
from oracle import scf_ref
from oracle import setup_ref as S
from oracle import workloads_ref as WR


def test_gaussian_form_factor_is_the_closed_form():
    # rho(r) = Z exp(-(r/R)^2) / (pi^(3/2) R^3) has the transform Z exp(-q^2 R^2 / 4)
    for z, radius in ((4.0, 1.0), (3.0, 0.8)):
        p = O.gaussian_pseudo(z, 0.45, rho_radius=radius)
        q = np.linspace(0.0, 12.0, 97)
        vol = 270.0
        got = O.atomic_charge_transform(p, vol, q)
        want = z * np.exp(-q * q * radius * radius / 4.0) / vol
        assert np.max(np.abs(got - want)) <= 1e-13 * z / vol
        assert got[0] == pytest.approx(z / vol, rel=1e-14)


def test_grid_density_matches_the_oracle():
    w, c = W.si2_gamma_atomic(), WR.si2_atomic()
    n = w.start_density()
    ref = S.atomic_density(c.cell, c.ecut_ha, c.dims(), c.species())
    assert n.shape == tuple(w.dims()) and n.flags.c_contiguous
    assert np.max(np.abs(n - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.min(n) >= 0.0
    assert float(n.sum()) * w.volume / n.size == pytest.approx(8.0, rel=1e-13)


def test_uniform_start_without_an_atomic_charge():
    # refstart.rs:56-59, 708-710: no PP_RHOATOM, an all-zero one, or one of the wrong
    # length means the uniform start
    assert W.si2_gamma().start_density() is None
    p = O.gaussian_pseudo(4.0, 0.45)
    assert not O.has_atomic_charge(p)
    p.rho_atom = np.zeros_like(p.r)
    assert not O.has_atomic_charge(p)
    p.rho_atom = np.ones(len(p.r) - 1)
    assert not O.has_atomic_charge(p)
    p.rho_atom = O.gaussian_pseudo(4.0, 0.45, rho_radius=1.0).rho_atom
    assert O.has_atomic_charge(p)
    # one species without a charge makes the whole start uniform
    w = W.si2_gamma_atomic()
    mixed = [w.species[0], O.Species(O.gaussian_pseudo(4.0, 0.45), np.zeros((1, 3)))]
    assert O.atomic_density(w.rows, w.ecut_ha, w.dims(), mixed) is None


def test_argument_checks():
    p = O.gaussian_pseudo(4.0, 0.45, rho_radius=1.0)
    with pytest.raises(L.BaandiError):
        O.atomic_charge_transform(p, 100.0, np.array([-1.0]))
    with pytest.raises(L.BaandiError):
        O.atomic_charge_transform(p, 0.0, np.array([1.0]))
    p.rho_atom = p.rho_atom.copy()
    p.rho_atom[5] = math.nan
    with pytest.raises(L.BaandiError) as e:
        O.atomic_charge_transform(p, 100.0, np.array([1.0]))
    assert e.value.code == L.BG_ENONFINITE


def test_oracle_scf_from_the_atomic_start():
    """Si2 Gamma to 1e-8 Ha (Fermi-Dirac 0.01 Ha): the atomic start reaches the uniform
    start's energy, with a first-map residual far below the uniform one; the converged
    spectrum has a threefold level holding the fourth band, so fixed occupations (four
    bands filled) would fill one of three degenerate states, whatever the start."""
    c = WR.si2_atomic()
    w = W.si2_gamma()
    pw = w.plane_waves()
    starts = [w.random_block(pw.npw, w.bands, seed_offset=100, real=True)]
    sp = c.species()
    n0 = S.atomic_density(c.cell, c.ecut_ha, c.dims(), sp)
    args = (c.rows, sp, c.ecut_ha, c.dims(), c.kpoints, True, c.bands, c.ionic_potential(), starts,
            O.ewald(w.rows, w.species))
    uni = scf_ref.run(*args, threshold_ha=1e-8, smearing_ha=0.01)
    atom = scf_ref.run(*args, threshold_ha=1e-8, smearing_ha=0.01, start_density=n0)
    assert uni.converged and atom.converged
    assert abs(atom.energy - uni.energy) <= 1e-7 * 2
    assert atom.dr2[0] < 0.2 * uni.dr2[0]
    e = np.sort(atom.eigenvalues[0])
    assert np.ptp(e[3:6]) < 1e-4 and e[2] < e[3] - 0.1 and e[6] > e[5] + 0.05
