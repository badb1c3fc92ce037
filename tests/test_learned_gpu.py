"""The learned preconditioner on the GPU: training samples, loss and gradient and the
Adam step against the FP64 oracle; the start network is TPA bit for bit; a network
trained on displaced Si2 geometries against TPA on a held-out geometry; the TPA
fallback; argument checks."""
import numpy as np
import pytest

from baandi_b200 import davidson as DV
from baandi_b200 import learned as LP
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import SolverError
from oracle import learned_ref as R

pytestmark = pytest.mark.gpu

AMP = 0.25   # Bohr: seeded displacement of every atom
TRAIN_SEEDS = range(8)
HELD_OUT = 100


@pytest.fixture(scope="module")
def problems(ctx):
    base = W.si2_gamma()
    train = [LP.exact_problem(LP.displaced(base, s, AMP), ctx, 8, 16) for s in TRAIN_SEEDS]
    hold_w = LP.displaced(base, HELD_OUT, AMP)
    return train, LP.exact_problem(hold_w, ctx, 8, 16), hold_w


def _one_state(ctx, p, it=2):
    (x, hx, lam), = LP.davidson_states(p, (it,))
    e = LP.ideal_corrections(p, x)
    s = LP.Samples(x.size, x.shape[1])
    s.add_state(ctx, x, hx, e, p.kinetic, lam)
    return s, R.samples(x, hx, e, p.kinetic, lam)


def _host(s):
    z = s.z.cpu().numpy()
    return (s.feats.cpu().numpy().astype(np.float64), s.base.cpu().numpy().astype(np.float64),
            s.a.cpu().numpy().astype(np.float64), z[:, 0] + 1j * z[:, 1], s.col.cpu().numpy(), s.ecol.cpu().numpy())


def test_samples_match_oracle(ctx, problems):
    s, ref = _one_state(ctx, problems[0][0])
    feats, base, a, z, col, ecol = _host(s)
    assert np.max(np.abs(feats - ref[0])) < 1e-6            # FP32 inputs of O(10)
    assert np.max(np.abs(base - ref[1])) < 1e-7
    assert np.max(np.abs(a - ref[2]) / np.maximum(ref[2], 1e-30)) < 1e-6
    assert np.max(np.abs(z - ref[3])) <= 1e-6 * np.max(np.abs(ref[3]))
    assert np.array_equal(col, ref[4])
    assert np.max(np.abs(ecol - ref[5]) / ref[5]) < 1e-12


def test_loss_and_gradient_match_oracle(ctx, problems):
    s, _ = _one_state(ctx, problems[0][0])
    rng = np.random.default_rng(2)
    p = LP.init_params(3)
    p[LP.OW3:LP.OB3] = rng.normal(0, 0.3, LP.N_HID).astype(np.float32)
    p[LP.OB3] = 0.1
    t = LP.Trainer(ctx, p)
    loss = t.loss_grad(s)
    g = t.grad.cpu().numpy().astype(np.float64)
    rl, rg = R.loss_grad(LP.from_bf16_bits(LP.to_bf16_bits(p)).astype(np.float64), *_host(s))
    assert abs(loss - rl) <= 1e-6 * abs(rl)
    assert np.linalg.norm(g - rg) <= 1e-5 * np.linalg.norm(rg)   # FP32 accumulation


def test_adam_step_matches_numpy(ctx, problems):
    s, _ = _one_state(ctx, problems[0][0])
    p = LP.init_params(4)
    t = LP.Trainer(ctx, p, lr=1e-2)
    t.step(s)
    g = t.grad.cpu().numpy().astype(np.float64)
    m1, m2 = 0.1 * g, 0.001 * g * g
    want = p - 1e-2 * (m1 / 0.1) / (np.sqrt(m2 / 0.001) + 1e-8)
    got = t.params()
    assert np.max(np.abs(got - want)) <= 1e-6 * max(1.0, np.max(np.abs(want)))
    assert np.array_equal(t.net.cpu().numpy().view(np.uint16), LP.to_bf16_bits(got))


def test_start_network_is_tpa_exactly(ctx, problems):
    _, hp, _ = problems
    o = DV.Options(8, 1e-8, 4, max_iterations=40, preconditioner="tpa")
    a = DV.solve(hp.op, hp.start, hp.kinetic, o)
    LP.install(ctx, LP.init_params(0))
    o.preconditioner = "learned"
    b = DV.solve(hp.op, hp.start, hp.kinetic, o)
    assert np.array_equal(a.eigenvalues, b.eigenvalues)
    assert (a.iterations, a.h_columns) == (b.iterations, b.h_columns)


@pytest.fixture(scope="module")
def trained(ctx, problems):
    """The network trained on the 8 displaced geometries (600 Adam steps) and the
    held-out correction loss before and after."""
    train, hp, _ = problems
    samples = LP.build_samples(ctx, train)
    held = LP.build_samples(ctx, [hp])
    t = LP.Trainer(ctx, LP.init_params(0), lr=3e-3)
    before = t.loss_grad(held)
    for _ in range(600):
        t.step(samples)
    return t.params(), before, t.loss_grad(held)


def test_trained_network_against_tpa_on_a_held_out_geometry(ctx, problems, trained):
    """Trained on 8 displaced Si2 geometries; on a ninth it lowers the correction loss
    and the H columns the Davidson needs (occupied bands to 1e-8 Ha, four seeded
    starts) against TPA, and reaches the same occupied eigenvalues."""
    train, hp, hold_w = problems
    params, before, after = trained
    assert after < 0.95 * before, (before, after)
    LP.install(ctx, params)
    cols = {"tpa": 0, "learned": 0}
    for so in (7, 11, 12, 13):
        start = hold_w.random_block(hp.op.global_len(), 8, seed_offset=so, real=True)
        res = {}
        for name in cols:
            o = DV.Options(8, 1e-8, 4, max_iterations=120, preconditioner=name)
            res[name] = DV.solve(hp.op, start, hp.kinetic, o)
            cols[name] += res[name].h_columns
            assert np.max(np.abs(res[name].eigenvalues[:4] - hp.evals[:4])) < 1e-7
    print(f"held-out loss {before:.4f} -> {after:.4f}; H columns tpa {cols['tpa']} learned {cols['learned']}")
    assert cols["learned"] < cols["tpa"]


def test_bad_network_falls_back_to_tpa(ctx, problems):
    _, hp, _ = problems
    bad = LP.init_params(0)
    bad[LP.OW3:LP.OB3] = np.random.default_rng(9).normal(0.0, 50.0, LP.N_HID)   # row-to-row multipliers e^(+-3)
    LP.install(ctx, bad)
    o = DV.Options(8, 1e-8, 4, max_iterations=120, preconditioner="learned")
    sol = DV.solve(hp.op, hp.start, hp.kinetic, o)
    assert sol.fallbacks == 1
    assert np.max(np.abs(sol.eigenvalues[:4] - hp.evals[:4])) < 1e-7


def test_learned_argument_checks(ctx, problems):
    _, hp, _ = problems
    LP.clear(ctx)
    with pytest.raises(SolverError):
        DV.solve(hp.op, hp.start, hp.kinetic, DV.Options(8, 1e-8, 4, preconditioner="learned"))
    p = LP.init_params(0)
    p[7] = np.nan
    with pytest.raises(SolverError):
        LP.install(ctx, p)


def test_complex_samples_and_gradient_match_oracle(ctx):
    """Complex rows (a Si8 k point): samples, loss and gradient against the oracle, with a
    seeded target in place of the exact correction (parity does not need the spectrum)."""
    from baandi_b200.hamiltonian import ComplexHamiltonian
    w = W.si8_k444()
    pw = w.plane_waves(w.kpoints[3][0])
    op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 8, ctx)
    op.set_owned_potential(w.ionic_potential(), 1)
    x = w.random_block(pw.npw, 6, seed_offset=21)
    hx = op.apply_block(x)
    lam = np.real(np.sum(np.conj(x) * hx, axis=0))
    e = 1e-3 * w.random_block(pw.npw, 6, seed_offset=22)
    kin = op.kinetic_diagonal()
    s = LP.Samples(x.size, 6)
    s.add_state(ctx, x, hx, e, kin, lam)
    ref = R.samples(x, hx, e, kin, lam)
    feats, base, a, z, col, ecol = _host(s)
    assert np.max(np.abs(feats - ref[0])) < 1e-6
    assert np.max(np.abs(base - ref[1])) < 1e-7
    assert np.max(np.abs(z - ref[3])) <= 1e-6 * np.max(np.abs(ref[3]))
    assert np.max(np.abs(ecol - ref[5]) / ref[5]) < 1e-12
    rng = np.random.default_rng(8)
    p = LP.init_params(5)
    p[LP.OW3:LP.OB3] = rng.normal(0, 0.3, LP.N_HID).astype(np.float32)
    t = LP.Trainer(ctx, p)
    loss = t.loss_grad(s)
    rl, rg = R.loss_grad(LP.from_bf16_bits(LP.to_bf16_bits(p)).astype(np.float64), feats, base, a, z, col, ecol)
    assert abs(loss - rl) <= 1e-6 * abs(rl)
    assert np.linalg.norm(t.grad.cpu().numpy() - rg) <= 1e-5 * np.linalg.norm(rg)


def test_start_network_is_tpa_on_a_complex_operator(ctx):
    from baandi_b200.hamiltonian import ComplexHamiltonian
    w = W.si8_k444()
    pw = w.plane_waves(w.kpoints[5][0])
    op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 48, ctx)
    op.set_owned_potential(w.ionic_potential(), 1)
    start = w.random_block(pw.npw, 24, seed_offset=3)
    kin = op.kinetic_diagonal()
    o = DV.Options(24, 1e-6, 16, max_iterations=8, preconditioner="tpa")
    a = DV.solve(op, start, kin, o)
    LP.install(ctx, LP.init_params(0))
    o.preconditioner = "learned"
    b = DV.solve(op, start, kin, o)
    assert np.array_equal(a.eigenvalues, b.eigenvalues)
    assert (a.iterations, a.h_columns) == (b.iterations, b.h_columns)


# ---- the batched solver (bg_kset_davidson_solve), the one the SCF runs

def _kset_solve(ctx, hp, start, name, its=120):
    from baandi_b200.hamiltonian import KPointSet
    ks = KPointSet([hp.op], ctx)
    o = DV.Options(8, 1e-8, 4, max_iterations=its, preconditioner=name)
    (sol,) = DV.solve_kset(ks, [start], [hp.kinetic], o)
    return sol


def test_kset_start_network_is_tpa_exactly(ctx, problems):
    _, hp, _ = problems
    a = _kset_solve(ctx, hp, hp.start, "tpa", 40)
    LP.install(ctx, LP.init_params(0))
    b = _kset_solve(ctx, hp, hp.start, "learned", 40)
    assert np.array_equal(a.eigenvalues, b.eigenvalues)
    assert (a.iterations, a.h_columns) == (b.iterations, b.h_columns)


def test_kset_trained_network_against_tpa(ctx, problems, trained):
    """The batched solver with the trained network on the held-out geometry: fewer H
    columns than TPA over four seeded starts, the same occupied eigenvalues."""
    _, hp, hold_w = problems
    LP.install(ctx, trained[0])
    cols = {"tpa": 0, "learned": 0}
    for so in (7, 11, 12, 13):
        start = hold_w.random_block(hp.op.global_len(), 8, seed_offset=so, real=True)
        for name in cols:
            sol = _kset_solve(ctx, hp, start, name)
            cols[name] += sol.h_columns
            assert np.max(np.abs(sol.eigenvalues[:4] - hp.evals[:4])) < 1e-7
    print(f"batched solver, H columns tpa {cols['tpa']} learned {cols['learned']}")
    assert cols["learned"] < cols["tpa"]


def test_kset_bad_network_falls_back_to_tpa(ctx, problems):
    _, hp, _ = problems
    bad = LP.init_params(0)
    bad[LP.OW3:LP.OB3] = np.random.default_rng(9).normal(0.0, 50.0, LP.N_HID)
    LP.install(ctx, bad)
    sol = _kset_solve(ctx, hp, hp.start, "learned")
    assert sol.fallbacks == 1
    assert np.max(np.abs(sol.eigenvalues[:4] - hp.evals[:4])) < 1e-7


def test_kset_learned_needs_a_network(ctx, problems):
    _, hp, _ = problems
    LP.clear(ctx)
    with pytest.raises(SolverError):
        _kset_solve(ctx, hp, hp.start, "learned", 5)
