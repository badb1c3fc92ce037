"""Ewald ion-ion energy: the host restatement (bg_setup_ewald) against the Madelung
constant of the simple cubic lattice in a neutralising background, against the
oracle's independent sum at other splitting parameters, and on the benchmark cells."""
import numpy as np

from baandi_b200 import operands as O
from baandi_b200 import systems as W
from oracle import ewald_ref as E

MADELUNG_SC = 2.8372974794806  # simple cubic Wigner lattice: E = -alpha Z^2 / (2 a)


def test_simple_cubic_madelung():
    for a in (1.0, 7.3):
        e = O.ewald(np.diag([a, a, a]), [O.Species(O.gaussian_pseudo(1.0, 0.5), np.zeros((1, 3)))])
        assert abs(e - (-MADELUNG_SC / (2 * a))) < 1e-12 / a
        for eta in (0.7 / a, 3.0 / a):
            assert abs(E.energy(np.diag([a, a, a]), np.zeros((1, 3)), [1.0], eta=eta) - e) < 1e-12 / a


def test_benchmark_cells_match_oracle():
    for name in ("si2", "si8", "al32"):
        w = W.WORKLOADS[name]()
        e = O.ewald(w.rows, w.species)
        pos = np.concatenate([np.atleast_2d(s.positions) for s in w.species])
        z = np.concatenate([np.full(len(np.atleast_2d(s.positions)), s.pseudo.z) for s in w.species])
        ref = E.energy(w.rows, pos, z, eta=1.3 * np.sqrt(np.pi) / abs(np.linalg.det(w.rows)) ** (1 / 3))
        assert abs(e - ref) < 1e-9 * abs(ref), (name, e, ref)
