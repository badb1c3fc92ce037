"""GPU block Davidson (bg_davidson_solve through the C ABI) against the reference's
dense fixture recipe, the dense eigensolver and the oracle's Davidson restatement
(FP64: eigenvalues within 1e-8 Ha of the oracle, 1e-11 on the dense fixture)."""
import numpy as np
import pytest

from baandi_b200 import davidson as DV
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian, DenseOperator, RealGammaHamiltonian
from oracle import davidson_ref as D
from tests.helpers import oracle_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cluster", [False, True])
def test_dense_fixture_real(ctx, cluster):
    """crates/dft-solvers/tests/ref_davidson.rs:113-228 on the GPU solver."""
    dim, bands, occupied = 32, 8, 6
    h = D.dct_fixture(dim, cluster)
    exact, q = np.linalg.eigh(h)
    op = DenseOperator(h, dim)
    opts = DV.Options(bands, 1e-13, occupied, first_step=True, max_iterations=400)
    sol = DV.solve(op, D.dct_start(dim, bands), np.diag(h).copy(), opts)
    assert sol.converged.all()
    assert np.max(np.abs(sol.eigenvalues - exact[:bands])) < 1e-11
    assert D.projector_error(sol.eigenvectors, q, occupied) < 2e-6
    assert sol.contractions > 0
    assert sol.h_columns == bands + (sol.h_columns - bands)
    ref = D.solve(lambda x: h @ x, D.dct_start(dim, bands), np.diag(h).copy(),
                  D.Options(bands, 1e-13, occupied, first_step=True, max_iterations=400))
    assert np.max(np.abs(sol.eigenvalues - ref.eigenvalues)) < 1e-11


def test_dense_fixture_complex(ctx):
    """A Hermitian analogue of the fixture (complex phases on the DCT basis)."""
    dim, bands, occupied = 40, 10, 7
    h = D.dct_fixture(dim, True).astype(np.complex128)
    ph = np.exp(1j * 0.37 * np.arange(dim))
    h = (ph[:, None] * h) * np.conj(ph)[None, :]
    exact, q = np.linalg.eigh(h)
    start = D.dct_start(dim, bands) * ph[:, None]
    op = DenseOperator(h, dim)
    sol = DV.solve(op, start, np.diag(h).real.copy(), DV.Options(bands, 1e-13, occupied, first_step=True,
                                                                  max_iterations=400))
    assert sol.converged.all()
    assert np.max(np.abs(sol.eigenvalues - exact[:bands])) < 1e-11
    assert D.projector_error(sol.eigenvectors, q, occupied) < 2e-6


def test_si2_gamma_real_vs_dense(ctx):
    """Si2 Gamma ORC path: 8 bands to 1e-10 Ritz change vs the exact dense spectrum."""
    from oracle import oracle as OR
    from oracle import setup_ref as S
    w = W.si2_gamma()
    pw = w.plane_waves()
    nl = w.nonlocal_table(pw)
    dims = w.dims()
    v = w.ionic_potential()
    op = RealGammaHamiltonian.new_owned(pw, dims, nl, 16, ctx)
    op.set_owned_potential(v, 1)
    n = pw.npw
    diag = op.diagonal_static() + v.mean()
    start = w.random_block(n, 8, real=True)
    sol = DV.solve(op, start, diag, DV.Options(8, 1e-10, 4, first_step=True, max_iterations=200))
    assert sol.converged.all()
    cell, b, onl = oracle_inputs(w, (0, 0, 0))
    plus, minus, _ = S.half_sphere(b)
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    H = OR.apply_gamma(dims, idx, plus, minus, v, S.orc_kinetic(plus, b.kpg2), S.orc_projectors(plus, onl.table), onl,
                       np.eye(n))
    exact = np.linalg.eigvalsh(0.5 * (H + H.T))[:8]
    assert np.max(np.abs(sol.eigenvalues - exact)) < 1e-8
    hx = op.apply_block(sol.eigenvectors)
    res = np.linalg.norm(hx - sol.eigenvectors * sol.eigenvalues[None, :], axis=0)
    assert np.max(res) < 1e-4


def test_si8_kpoint_vs_oracle_davidson(ctx):
    """One k point of Si8 (complex path, 24 bands): GPU Davidson vs the oracle's
    Davidson on the oracle's apply, same start and options."""
    from oracle import oracle as OR
    from oracle import setup_ref as S
    w = W.si8_k444()
    k = w.kpoints[3][0]
    pw = w.plane_waves(k)
    nl = w.nonlocal_table(pw)
    dims = w.dims()
    v = w.ionic_potential()
    op = ComplexHamiltonian.new_owned(pw, dims, nl, 48, ctx)
    op.set_owned_potential(v, 1)
    diag = op.diagonal_static() + v.mean()
    start = w.random_block(pw.npw, 24, seed_offset=7)
    opts = DV.Options(24, 1e-9, 16, first_step=True, max_iterations=60)
    sol = DV.solve(op, start, diag, opts)
    cell, b, onl = oracle_inputs(w, k)
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    ref = D.solve(lambda x: OR.apply_complex(dims, idx, v, 0.5 * b.kpg2, onl, x), start, diag,
                  D.Options(24, 1e-9, 16, first_step=True, max_iterations=60))
    assert sol.converged.all() and ref.converged.all()
    assert np.max(np.abs(sol.eigenvalues - ref.eigenvalues)) < 1e-8


def test_invalid_options(ctx):
    h = D.dct_fixture(16, False)
    op = DenseOperator(h, 16)
    from baandi_b200.hamiltonian import SolverError
    with pytest.raises(SolverError):
        DV.solve(op, D.dct_start(16, 4), np.diag(h).copy(), DV.Options(4, -1.0, 2))
    with pytest.raises(SolverError):
        DV.solve(op, D.dct_start(16, 4), np.diag(h).copy(), DV.Options(4, 1e-8, 5))
    bad = D.dct_start(16, 4)
    bad[0, 0] = np.nan
    with pytest.raises(SolverError):
        DV.solve(op, bad, np.diag(h).copy(), DV.Options(4, 1e-8, 2))
