"""The device-driven Davidson over a k-point set (bg_kset_davidson_solve): every k point
runs the reference Davidson (crates/dft-solvers/src/ref_davidson.rs:117-366,
ref_davidson_complex.rs:641-1110) with its reduced problem and control logic on the
GPU.  Checked against the reference's dense fixture and the exact spectrum, against the
host-driven solver (bg_davidson_solve) on the same operators and starts, and graph
replay against direct launches (bitwise)."""
import numpy as np
import pytest

from baandi_b200 import davidson as DV
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian, DenseOperator, KPointSet, RealGammaHamiltonian, SolverError
from oracle import davidson_ref as D

pytestmark = pytest.mark.gpu


def _dense_pair(cluster_a, cluster_b, dim, bands, complex_=False):
    hs = [D.dct_fixture(dim, cluster_a), D.dct_fixture(dim, cluster_b)]
    starts = [D.dct_start(dim, bands), D.dct_start(dim, bands)]
    if complex_:
        ph = np.exp(1j * 0.37 * np.arange(dim))
        hs = [(ph[:, None] * h.astype(np.complex128)) * np.conj(ph)[None, :] for h in hs]
        starts = [s * ph[:, None] for s in starts]
    return hs, starts


@pytest.mark.parametrize("complex_", [False, True])
def test_dense_fixture_pair(ctx, complex_):
    """crates/dft-solvers/tests/ref_davidson.rs:113-228 for two fixtures (plain and
    clustered spectrum) solved together: roots to 1e-11, occupied projectors to 2e-6,
    contractions exercised, and the same answer as the host-driven solver."""
    dim, bands, occupied = 32, 8, 6
    hs, starts = _dense_pair(False, True, dim, bands, complex_)
    ops = [DenseOperator(h, dim, ctx) for h in hs]
    ks = KPointSet(ops, ctx)
    opts = DV.Options(bands, 1e-13, occupied, first_step=True, max_iterations=400)
    diags = [np.diag(h).real.copy() for h in hs]
    sols = DV.solve_kset(ks, starts, diags, opts)
    for h, op, x0, dg, sol in zip(hs, ops, starts, diags, sols):
        exact, q = np.linalg.eigh(h)
        assert sol.converged.all()
        assert np.max(np.abs(sol.eigenvalues - exact[:bands])) < 1e-11
        assert D.projector_error(sol.eigenvectors, q, occupied) < 2e-6
        assert sol.contractions > 0
        host = DV.solve(op, x0, dg, opts)
        assert np.max(np.abs(sol.eigenvalues - host.eigenvalues)) < 1e-12
        assert abs(sol.iterations - host.iterations) <= 1


def test_graph_replay_equals_direct_launches(ctx):
    dim, bands = 32, 8
    hs, starts = _dense_pair(True, False, dim, bands)
    ks = KPointSet([DenseOperator(h, dim, ctx) for h in hs], ctx)
    opts = DV.Options(bands, 1e-12, 6, first_step=False, max_iterations=200)
    diags = [np.diag(h).copy() for h in hs]
    a = DV.solve_kset(ks, starts, diags, opts, graph=True)
    b = DV.solve_kset(ks, starts, diags, opts, graph=False)
    for x, y in zip(a, b):
        assert np.array_equal(x.eigenvalues, y.eigenvalues)
        assert np.array_equal(x.eigenvectors, y.eigenvectors)
        assert x.iterations == y.iterations and x.h_columns == y.h_columns


def _si8_set(ctx, kidx, bands=24):
    w = W.si8_k444()
    v = w.ionic_potential()
    ops, starts, diags = [], [], []
    for i, kk in enumerate(kidx):
        k = w.kpoints[kk][0]
        pw = w.plane_waves(k)
        op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 2 * bands, ctx)
        op.set_owned_potential(v, 1)
        ops.append(op)
        starts.append(w.random_block(pw.npw, bands, seed_offset=20 + i))
        diags.append(op.diagonal_static() + v.mean())
    return ops, starts, diags


def test_si8_kset_matches_single_solves(ctx):
    """Four Si8 k points (uneven plane-wave counts) at once vs one host-driven solve
    per k point: eigenvalues within 1e-9 Ha, every band converged."""
    ops, starts, diags = _si8_set(ctx, [0, 5, 17, 35])
    ks = KPointSet(ops, ctx)
    opts = DV.Options(24, 1e-9, 16, first_step=True, max_iterations=60)
    sols = DV.solve_kset(ks, starts, diags, opts)
    for op, x0, dg, sol in zip(ops, starts, diags, sols):
        host = DV.solve(op, x0, dg, opts)
        assert sol.converged.all() and host.converged.all()
        assert np.max(np.abs(sol.eigenvalues - host.eigenvalues)) < 1e-9
        hx = op.apply_block(sol.eigenvectors)
        res = np.linalg.norm(hx - sol.eigenvectors * sol.eigenvalues[None, :], axis=0)
        assert np.max(res) < 1e-3
        gram = sol.eigenvectors.conj().T @ sol.eigenvectors
        assert np.max(np.abs(gram - np.eye(24))) < 1e-10


def test_si2_gamma_kset(ctx):
    w = W.si2_gamma()
    pw = w.plane_waves()
    v = w.ionic_potential()
    op = RealGammaHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 16, ctx)
    op.set_owned_potential(v, 1)
    diag = op.diagonal_static() + v.mean()
    start = w.random_block(pw.npw, 8, real=True)
    opts = DV.Options(8, 1e-10, 4, first_step=True, max_iterations=200)
    (sol,) = DV.solve_kset(KPointSet([op], ctx), [start], [diag], opts)
    host = DV.solve(op, start, diag, opts)
    assert sol.converged.all()
    assert np.max(np.abs(sol.eigenvalues - host.eigenvalues)) < 1e-9


def test_kset_errors(ctx):
    dim, bands = 24, 4
    h = D.dct_fixture(dim, False)
    ks = KPointSet([DenseOperator(h, dim, ctx), DenseOperator(h, dim, ctx)], ctx)
    x = D.dct_start(dim, bands)
    dep = x.copy()
    dep[:, 1] = dep[:, 0]
    opts = DV.Options(bands, 1e-10, 2, max_iterations=50)
    with pytest.raises(SolverError) as e:
        DV.solve_kset(ks, [x, dep], [np.diag(h).copy()] * 2, opts)
    assert "numerically dependent" in str(e.value) and "k point 1" in str(e.value)
    bad = x.copy()
    bad[0, 0] = np.inf
    with pytest.raises(SolverError):
        DV.solve_kset(ks, [bad, x], [np.diag(h).copy()] * 2, opts)
    with pytest.raises(SolverError):
        DV.solve_kset(ks, [x, x], [np.diag(h).copy()] * 2, DV.Options(bands, 1e-10, 5))
    sols = DV.solve_kset(ks, [x, x], [np.diag(h).copy()] * 2, opts)  # usable after the errors
    assert all(s.converged.all() for s in sols)


@pytest.mark.parametrize("kind", ["tpa", "ritz_shift"])
def test_preconditioner_variants_vs_oracle(ctx, kind):
    """The TPA and Ritz-shift corrections of the preconditioner seam
    (crates/dft-solvers/src/lib.rs:176-309) in both GPU solvers against the oracle
    Davidson with the same correction on Si2 Gamma: eigenvalues within 1e-8 Ha."""
    from oracle import oracle as OR
    from oracle import setup_ref as S
    from tests.helpers import oracle_inputs
    w = W.si2_gamma()
    pw = w.plane_waves()
    v = w.ionic_potential()
    dims = w.dims()
    op = RealGammaHamiltonian.new_owned(pw, dims, w.nonlocal_table(pw), 16, ctx)
    op.set_owned_potential(v, 1)
    diag = op.kinetic_diagonal() if kind == "tpa" else op.diagonal_static() + v.mean()
    start = w.random_block(pw.npw, 8, real=True)
    opts = DV.Options(8, 1e-10, 4, first_step=True, max_iterations=200, preconditioner=kind)
    single = DV.solve(op, start, diag, opts)
    (batched,) = DV.solve_kset(KPointSet([op], ctx), [start], [diag], opts)
    cell, b, onl = oracle_inputs(w, (0, 0, 0))
    plus, minus, _ = S.half_sphere(b)
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    korc, porc = S.orc_kinetic(plus, b.kpg2), S.orc_projectors(plus, onl.table)
    ref = D.solve(lambda x: OR.apply_gamma(dims, idx, plus, minus, v, korc, porc, onl, x), start, diag,
                  D.Options(8, 1e-10, 4, first_step=True, max_iterations=200, preconditioner=kind))
    assert single.converged.all() and batched.converged.all() and ref.converged.all()
    assert np.max(np.abs(single.eigenvalues - ref.eigenvalues)) < 1e-8
    assert np.max(np.abs(batched.eigenvalues - ref.eigenvalues)) < 1e-8
    assert abs(single.iterations - ref.iterations) <= 2
