"""Committed golden fixtures (tests/golden/make_golden.py): the oracle reproduces them
(CPU), and the CUDA path matches them through the C ABI (GPU, <= 1e-12 per column)."""
import os

import numpy as np
import pytest

from baandi_b200 import systems as W
from oracle import davidson_ref as D
from oracle import oracle as OR
from oracle import setup_ref as S
from tests.helpers import colwise_rel, oracle_inputs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def test_oracle_reproduces_si2_golden():
    g = _load("si2_apply.npz")
    w = W.si2_gamma()
    cell, b, nl = oracle_inputs(w, (0, 0, 0))
    assert np.array_equal(b.miller, g["miller"])
    dims = [int(d) for d in g["dims"]]
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    yc = OR.apply_complex(dims, idx, g["v"], 0.5 * b.kpg2, nl, g["xc"])
    assert colwise_rel(yc, g["yc"]) < 1e-14
    plus, minus, _ = S.half_sphere(b)
    yr = OR.apply_gamma(dims, idx, plus, minus, g["v"], S.orc_kinetic(plus, b.kpg2), S.orc_projectors(plus, nl.table),
                        nl, g["xr"])
    assert colwise_rel(yr, g["yr"]) < 1e-14


def test_oracle_davidson_golden():
    g = _load("dct_davidson.npz")
    h = g["h"]
    sol = D.solve(lambda x: h @ x, g["start"], np.diag(h).copy(), D.Options(8, 1e-13, 6, True, 0, 400))
    assert np.max(np.abs(sol.eigenvalues - g["exact"])) < 1e-11


@pytest.mark.gpu
def test_cuda_matches_si2_golden(ctx):
    from baandi_b200.hamiltonian import ComplexHamiltonian, RealGammaHamiltonian
    g = _load("si2_apply.npz")
    w = W.si2_gamma()
    pw = w.plane_waves()
    assert np.array_equal(pw.miller, g["miller"])
    nl = w.nonlocal_table(pw)
    dims = [int(d) for d in g["dims"]]
    c = ComplexHamiltonian.new_owned(pw, dims, nl, 3, ctx)
    c.set_owned_potential(g["v"], 1)
    assert colwise_rel(c.apply_block(g["xc"]), g["yc"]) <= 1e-12
    r = RealGammaHamiltonian.new_owned(pw, dims, nl, 3, ctx)
    r.set_owned_potential(g["v"], 1)
    assert colwise_rel(r.apply_block(g["xr"]), g["yr"]) <= 1e-12
