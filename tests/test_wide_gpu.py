"""The reduced problem of the batched Davidson on many thread blocks (the path that
bg_kset_davidson_solve takes beyond capacity 128, the Gamma-only supercells' 320 and 960):
the generalised Hermitian eigensolve on its own (bg_reduced_eigh) against numpy on
clustered pencils up to m = 960, the solver with the many-block reduced problem against
the one-block control kernel and the reference's dense fixture, and a Si64 Davidson at
capacity 320 against the oracle Davidson (eigenvalues within 1e-8 Ha).

Reference: crates/dft-numerics/src/linalg.rs:234-444 (overlap factor, reduced solve),
crates/dft-solvers/src/ref_davidson_complex.rs:641-1110 (the complex Davidson)."""
import numpy as np
import pytest

from baandi_b200 import davidson as DV
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian, DenseOperator, KPointSet, RealGammaHamiltonian
from oracle import davidson_ref as D

pytestmark = pytest.mark.gpu


def _clustered_pencil(m, complex_, seed):
    """H with exact, near-degenerate (1e-10 apart) and well separated eigenvalue groups in
    a random unitary basis; S = I + a small positive perturbation (well conditioned)."""
    rng = np.random.default_rng(seed)
    lam = np.sort(rng.uniform(-2.0, 12.0, m))
    for start in range(0, m - 8, 37):       # clusters of 1 to 6 members
        size = 1 + start % 6
        lam[start:start + size] = lam[start] + 1e-10 * np.arange(size) * (start % 2)
    lam = np.sort(lam)
    if complex_:
        g = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
    else:
        g = rng.standard_normal((m, m))
    q, _ = np.linalg.qr(g)
    h = (q * lam[None, :]) @ q.conj().T
    h = 0.5 * (h + h.conj().T)
    b = rng.standard_normal((m, m)) + (1j * rng.standard_normal((m, m)) if complex_ else 0)
    s = np.eye(m) + 0.05 * (b @ b.conj().T) / m
    s = 0.5 * (s + s.conj().T)
    return h, s


@pytest.mark.parametrize("m,complex_", [(37, True), (320, False), (320, True), (960, True)])
def test_reduced_eigh_matches_numpy(ctx, m, complex_):
    h, s = _clustered_pencil(m, complex_, 7 + m)
    w, c, ms = DV.reduced_eigh(s, h, ctx)
    l = np.linalg.cholesky(s)
    li = np.linalg.inv(l)
    ref = np.linalg.eigvalsh(li @ h @ li.conj().T)
    scale = max(1.0, np.max(np.abs(ref)))
    assert np.max(np.abs(w - ref)) <= 1e-11 * scale
    gram = c.conj().T @ s @ c
    assert np.max(np.abs(gram - np.eye(m))) <= 1e-10
    res = h @ c - (s @ c) * w[None, :]
    assert np.max(np.abs(res)) <= 1e-10 * scale
    assert ms > 0.0


def test_reduced_eigh_rejects_dependent_overlap(ctx):
    from baandi_b200.hamiltonian import SolverError
    m = 64
    h, s = _clustered_pencil(m, True, 3)
    x = np.random.default_rng(1).standard_normal((m, 10))
    s = x @ x.T   # rank 10
    with pytest.raises(SolverError) as e:
        DV.reduced_eigh(s, h, ctx)
    assert "dependent" in str(e.value)


def _dense_pair(dim, bands):
    hs = [D.dct_fixture(dim, False), D.dct_fixture(dim, True)]
    ph = np.exp(1j * 0.37 * np.arange(dim))
    hs = [(ph[:, None] * h.astype(np.complex128)) * np.conj(ph)[None, :] for h in hs]
    starts = [D.dct_start(dim, bands) * ph[:, None] for _ in hs]
    return hs, starts


def test_dense_fixture_many_block_reduced_problem(ctx):
    """crates/dft-solvers/tests/ref_davidson.rs:113-228 with the reduced problem on many
    blocks: roots to 1e-11, contractions exercised, the same iterations as the one-block
    control kernel and eigenvalues equal to rounding."""
    dim, bands, occupied = 32, 8, 6
    hs, starts = _dense_pair(dim, bands)
    ks = KPointSet([DenseOperator(h, dim, ctx) for h in hs], ctx)
    opts = DV.Options(bands, 1e-13, occupied, first_step=True, max_iterations=400)
    diags = [np.diag(h).real.copy() for h in hs]
    wide = DV.solve_kset(ks, starts, diags, opts, reduced="wide")
    block = DV.solve_kset(ks, starts, diags, opts, reduced="block")
    for h, a, b in zip(hs, wide, block):
        exact, q = np.linalg.eigh(h)
        assert a.converged.all()
        assert np.max(np.abs(a.eigenvalues - exact[:bands])) < 1e-11
        assert D.projector_error(a.eigenvectors, q, occupied) < 2e-6
        assert a.contractions > 0
        assert np.max(np.abs(a.eigenvalues - b.eigenvalues)) < 1e-12
        assert abs(a.iterations - b.iterations) <= 1


def test_si8_kset_many_block_matches_one_block(ctx):
    w = W.si8_k444()
    v = w.ionic_potential()
    ops, starts, diags = [], [], []
    for i, kk in enumerate([0, 5, 17, 35]):
        k = w.kpoints[kk][0]
        pw = w.plane_waves(k)
        op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 48, ctx)
        op.set_owned_potential(v, 1)
        ops.append(op)
        starts.append(w.random_block(pw.npw, 24, seed_offset=20 + i))
        diags.append(op.diagonal_static() + v.mean())
    ks = KPointSet(ops, ctx)
    opts = DV.Options(24, 1e-9, 16, first_step=True, max_iterations=60)
    wide = DV.solve_kset(ks, starts, diags, opts, reduced="wide")
    block = DV.solve_kset(ks, starts, diags, opts, reduced="block")
    for a, b in zip(wide, block):
        assert a.converged.all() and b.converged.all()
        assert np.max(np.abs(a.eigenvalues - b.eigenvalues)) < 1e-9


def test_si2_gamma_real_many_block(ctx):
    w = W.si2_gamma()
    pw = w.plane_waves()
    v = w.ionic_potential()
    op = RealGammaHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 16, ctx)
    op.set_owned_potential(v, 1)
    diag = op.diagonal_static() + v.mean()
    start = w.random_block(pw.npw, 8, real=True)
    opts = DV.Options(8, 1e-10, 4, first_step=True, max_iterations=200)
    ks = KPointSet([op], ctx)
    (a,) = DV.solve_kset(ks, [start], [diag], opts, reduced="wide")
    (b,) = DV.solve_kset(ks, [start], [diag], opts, reduced="block")
    assert a.converged.all()
    assert np.max(np.abs(a.eigenvalues - b.eigenvalues)) < 1e-10


def test_si64_davidson_capacity_320_vs_oracle(ctx):
    """Si64 (Gamma, complex path, 23,847 plane waves, 256 projectors): 160 bands at
    capacity 320, the reduced problem on many blocks, against the oracle Davidson on the
    oracle's apply with the same start and options, 30 iterations each: the same bands
    converge, occupied eigenvalues within 1e-8 Ha, every eigenvalue within 1e-7 Ha, and the
    one-block reduced problem gives the same run."""
    from oracle import oracle as OR
    from oracle import setup_ref as S
    from tests.helpers import oracle_inputs
    w = W.si64_gamma()
    dims = w.dims()
    pw = w.plane_waves()
    v = w.ionic_potential()
    bands, occupied, its = 160, 128, 30
    op = ComplexHamiltonian.new_owned(pw, dims, w.nonlocal_table(pw), 2 * bands, ctx)
    op.set_owned_potential(v, 1)
    diag = op.diagonal_static() + v.mean()
    start = w.random_block(pw.npw, bands, seed_offset=5)
    opts = DV.Options(bands, 1e-9, occupied, first_step=False, max_iterations=its)
    ks = KPointSet([op], ctx)
    (sol,) = DV.solve_kset(ks, [start], [diag], opts)
    (blk,) = DV.solve_kset(ks, [start], [diag], opts, reduced="block")
    _, b, onl = oracle_inputs(w, (0.0, 0.0, 0.0))
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    ref = D.solve(lambda x: OR.apply_complex(dims, idx, v, 0.5 * b.kpg2, onl, x), start, diag,
                  D.Options(bands, 1e-9, occupied, first_step=False, max_iterations=its))
    assert sol.iterations == ref.iterations == blk.iterations
    assert abs(int(sol.converged.sum()) - int(ref.converged.sum())) <= 2
    assert np.max(np.abs(sol.eigenvalues[:occupied] - ref.eigenvalues[:occupied])) < 1e-8
    assert np.max(np.abs(sol.eigenvalues - ref.eigenvalues)) < 1e-7
    assert np.max(np.abs(sol.eigenvalues - blk.eigenvalues)) < 1e-8
    gram = sol.eigenvectors.conj().T @ sol.eigenvectors
    assert np.max(np.abs(gram - np.eye(bands))) < 1e-9
