"""Generate the committed golden fixtures of the Hamiltonian apply with the oracle.

    python tests/golden/make_golden.py

Writes tests/golden/si2_apply.npz: Si2 (fcc a = 10.26 Bohr, 30 Ry, 25^3 grid, synthetic
Si pseudopotential) complex and Gamma-ORC applies of seeded columns, with the operands'
fingerprints (Miller order, grid); and tests/golden/dct_davidson.npz: the reference's
dense Davidson fixture (32 x 32, clusters) with its exact lowest 8 eigenvalues.  The
fixtures pin the oracle between runs and are compared with the CUDA path on the GPU.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from baandi_b200 import systems as W  # noqa: E402
from oracle import davidson_ref as D  # noqa: E402
from oracle import oracle as OR  # noqa: E402
from oracle import setup_ref as S  # noqa: E402


def si2():
    w = W.si2_gamma()
    cell = S.Cell(w.rows)
    b = S.basis_at_k(cell, w.ecut_ha)
    p = w.species[0].pseudo
    ps = S.Pseudo(p.z, p.r, p.rab, p.local, [S.Projector(l, u) for l, u in zip(p.l, p.beta)], p.dij)
    nl = S.nonlocal_table(b, cell.volume, [S.Species(ps, w.species[0].positions)])
    dims, _ = S.grid_dims(cell, w.ecut_ha)
    v = w.ionic_potential()
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    xc = w.random_block(b.npw, 3, seed_offset=101)
    yc = OR.apply_complex(dims, idx, v, 0.5 * b.kpg2, nl, xc)
    plus, minus, _ = S.half_sphere(b)
    xr = w.random_block(b.npw, 3, seed_offset=102, real=True)
    yr = OR.apply_gamma(dims, idx, plus, minus, v, S.orc_kinetic(plus, b.kpg2), S.orc_projectors(plus, nl.table), nl,
                        xr)
    np.savez_compressed(os.path.join(HERE, "si2_apply.npz"), miller=b.miller, dims=np.array(dims), v=v, xc=xc, yc=yc,
                        xr=xr, yr=yr)


def dct():
    h = D.dct_fixture(32, True)
    np.savez_compressed(os.path.join(HERE, "dct_davidson.npz"), h=h, start=D.dct_start(32, 8),
                        exact=np.linalg.eigvalsh(h)[:8])


if __name__ == "__main__":
    si2()
    dct()
    print("wrote", os.listdir(HERE))
