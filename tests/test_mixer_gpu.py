"""GPU density mixer (bg_mixer_*) against the reference's own known answers
(crates/dft-engine/tests/refscf.rs) and against the oracle mixer on a long seeded
sequence on a density sphere's worth of coefficients."""
import math

import numpy as np
import pytest

from baandi_b200.hamiltonian import SolverError
from baandi_b200.mixer import Broyden, Profile
from oracle import broyden_ref as B

pytestmark = pytest.mark.gpu

MV = 1.0 / (8.0 * math.pi)


def test_closed_form_fixed_point(ctx):
    """refscf.rs:19-47: gamma = -27/97, next = (1, 93/97), then (1, 1)."""
    mix = Broyden([1.0, 1.0], [True, True], 1.0, 2.0, MV, Profile(beta=0.5), ctx)
    nxt, d = mix.update(np.zeros(2), [2.0, 3.0])
    assert np.array_equal(nxt, [1.0, 1.5]) and d.occupancy == 0 and d.inserted_slot is None
    x = nxt
    nxt, d = mix.update(x, [0.0, -1.5])
    assert d.occupancy == 1
    assert abs(mix.gamma()[0] + 27.0 / 97.0) < 1e-14
    assert abs(nxt[0].real - 1.0) < 1e-14 and abs(nxt[1].real - 93.0 / 97.0) < 1e-14
    x = nxt
    nxt, _ = mix.update(x, [2 - 2 * x[0].real, 3 - 3 * x[1].real])
    assert abs(nxt[0].real - 1.0) < 1e-14 and abs(nxt[1].real - 1.0) < 1e-14


def test_metric_and_reduced_residual(ctx):
    """refscf.rs:48-84 and :160-171."""
    m = Broyden([0.0, 1.0, 4.0, 9.0], [True, True, True, False], 1.0, 2.0, 2.0, Profile(), ctx)
    a = np.array([900, 1 + 2j, 2 - 1j, 40])
    b = np.array([-500, 3 - 1j, -1 + 2j, 70])
    assert abs(m.metric(a, b)) < 1e-13
    assert abs(m.metric(a, a) - 100 * math.pi) < 1e-12
    g2 = [1.0, 2.0, 4.0]
    mix = Broyden(g2, [True] * 3, 1.0, 2.0, MV, Profile(beta=0.5), ctx)
    f1 = np.array([2.0, -1.0, 0.5 + 0.25j])
    x, _ = mix.update(np.zeros(3), f1)
    assert np.array_equal(mix.reduced_residual(), f1)
    f2 = np.array([0.3, 0.7, -0.2 + 0.1j])
    mix.update(x, f2)
    red = mix.reduced_residual()
    df = f1 - f2
    assert np.max(np.abs(red - (f2 - mix.gamma()[0] * df))) < 1e-15
    assert abs(mix.metric(df, red)) < 1e-14 * max(mix.metric(f2, f2), 1.0)


def test_ring_eviction_and_thomas_fermi(ctx):
    """refscf.rs:117-158 (history 2) and :172-195 (Thomas-Fermi opt-in)."""
    mix = Broyden([1.0] * 3, [True] * 3, 1.0, 2.0, MV, Profile(beta=0.5, history=2), ctx)
    ref = B.Broyden([1.0] * 3, [True] * 3, 1.0, 2.0, MV, beta=0.5, history=2)
    f = np.array([3.0, 4.0, 5.0], complex)
    for k in range(7):
        if k > 0:
            f[(k - 1) % 3] -= 1.0
        x = np.array([k, k * k, k ** 3], complex)
        out, d = mix.update(x, f)
        want, dr = ref.update(x, f)
        assert d.occupancy == min(k, 2) and d.inserted_slot == dr["slot"]
        assert np.max(np.abs(out - want)) < 1e-12
    tf = Broyden([0.0, 1.0, 9.0], [True, True, False], 10.0, 2.0, MV, Profile(beta=0.7, thomas_fermi=True), ctx)
    out, _ = tf.update([2.0, 3.0, 4.0], [0.0, 1.0, 2.0])
    rs = (30.0 / (8.0 * math.pi)) ** (1 / 3)
    a = (12.0 / math.pi) ** (2 / 3) / rs
    assert out[0] == 2.0 and out[2] == 5.4
    assert abs(out[1].real - (3.0 + 0.7 / (1.0 + a))) < 1e-14


def test_singular_history_is_an_error(ctx):
    """refscf.rs:196-207: singular history is an error, and it ends the mixer."""
    mix = Broyden([1.0], [True], 1.0, 2.0, MV, Profile(), ctx)
    mix.update([0.0], [1.0])
    with pytest.raises(SolverError) as e:
        mix.update([1.0], [1.0])
    assert "singular Broyden history at iteration 2" in str(e.value)
    with pytest.raises(SolverError):
        mix.update([2.0], [0.5])


def test_long_sequence_matches_oracle(ctx):
    """A seeded nonlinear fixed-point iteration on 40,000 coefficients (a density
    sphere's size) with some non-smooth G: every update agrees with the oracle to
    1e-12 relative, or to 50 eps cond(A) once the history Gram A grows ill-conditioned
    (gamma = A^-1 b carries that amplification in any order of summation); history 8,
    so the ring wraps; host and device vectors agree bitwise."""
    import torch
    rng = np.random.default_rng(9)
    n = 40000
    g2 = np.sort(rng.uniform(0.0, 60.0, n))
    g2[0] = 0.0
    smooth = g2 < 40.0
    target = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / (1.0 + g2)
    stiff = 0.3 + g2 / (1.0 + g2)
    dev = Broyden(g2, smooth, 270.0, 32.0, 270.0, Profile(beta=0.4, history=8, thomas_fermi=True), ctx)
    host = Broyden(g2, smooth, 270.0, 32.0, 270.0, Profile(beta=0.4, history=8, thomas_fermi=True), ctx)
    ref = B.Broyden(g2, smooth, 270.0, 32.0, 270.0, beta=0.4, history=8, thomas_fermi=True)
    x = np.zeros(n, complex)
    xd = torch.zeros(n, dtype=torch.complex128, device="cuda")
    for it in range(14):
        f = stiff * (target - x) + 0.05 * np.tanh(x.real) * (1 + 0j)
        want, dr = ref.update(x, f)
        got, d = host.update(x, f)
        assert d.occupancy == dr["occupancy"]
        scale = np.max(np.abs(want))
        tol = 1e-12 if dr["condition"] is None else max(1e-12, 50 * np.finfo(float).eps * dr["condition"])
        if dr["condition"] is not None:
            c = dr["condition"]
            assert abs(d.condition - c) <= max(1e-6, 1e3 * np.finfo(float).eps * c) * c
        assert np.max(np.abs(got - want)) <= tol * scale, (it, dr["condition"])
        gd, _ = dev.update(xd, torch.from_numpy(f).cuda())
        assert np.array_equal(gd.cpu().numpy(), got)
        x = got
        xd = gd
