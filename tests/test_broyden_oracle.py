"""Pins of the mixer oracle (oracle/broyden_ref.py) against the reference's own
known-answer tests, crates/dft-engine/tests/refscf.rs (CPU only)."""
import math

import numpy as np
import pytest

from oracle import broyden_ref as B

MV = 1.0 / (8.0 * math.pi)  # metric volume of the reference tests: unit weights at G^2 = 1


def test_two_dimensional_linear_fixed_point_closed_form():
    """refscf.rs:19-47: F(x) = (2,3) - diag(2,3) x; gamma = -27/97, next = (1, 93/97),
    then the exact fixed point (1, 1)."""
    mix = B.Broyden([1.0, 1.0], [True, True], 1.0, 2.0, MV, beta=0.5)
    x = np.zeros(2, complex)
    nxt, d = mix.update(x, [2.0, 3.0])
    assert np.array_equal(nxt, [1.0, 1.5]) and d["occupancy"] == 0
    x = nxt
    nxt, d = mix.update(x, [0.0, -1.5])
    assert d["occupancy"] == 1
    assert abs(mix.gamma[0] + 27.0 / 97.0) < 1e-14
    assert abs(nxt[0].real - 1.0) < 1e-14 and abs(nxt[1].real - 93.0 / 97.0) < 1e-14
    x = nxt
    nxt, _ = mix.update(x, [2 - 2 * x[0].real, 3 - 3 * x[1].real])
    assert abs(nxt[0].real - 1.0) < 1e-14 and abs(nxt[1].real - 1.0) < 1e-14


def test_reduced_residual_is_metric_orthogonal():
    """refscf.rs:48-84: F~ = F - gamma dF is metric-orthogonal to dF."""
    g2 = [1.0, 2.0, 4.0]
    mix = B.Broyden(g2, [True] * 3, 1.0, 2.0, MV, beta=0.5)
    f1 = np.array([2.0, -1.0, 0.5 + 0.25j])
    x, _ = mix.update(np.zeros(3, complex), f1)
    assert np.array_equal(mix.reduced, f1)
    f2 = np.array([0.3, 0.7, -0.2 + 0.1j])
    mix.update(x, f2)
    df = f1 - f2
    w = B.metric_weights(MV, g2, [True] * 3)
    red = mix.reduced
    assert np.max(np.abs(red - (f2 - mix.gamma[0] * df))) < 1e-15
    assert abs(B.metric_dot(w, df, red)) < 1e-14 * max(B.metric_dot(w, f2, f2), 1.0)


def test_ring_eviction_keeps_last_two_secants():
    """refscf.rs:117-158: history 2, unit-vector differences: gamma is the matching
    component of F and the update is exact."""
    mix = B.Broyden([1.0] * 3, [True] * 3, 1.0, 2.0, MV, beta=0.5, history=2)
    f = np.array([3.0, 4.0, 5.0], complex)
    fs, xs = [], []
    for k in range(7):
        if k > 0:
            f[(k - 1) % 3] -= 1.0
        x = np.array([k, k * k, k ** 3], complex)
        out, d = mix.update(x, f)
        assert d["occupancy"] == min(k, 2)
        assert d["slot"] == ((k - 1) % 2 if k > 0 else None)
        expected = x + 0.5 * f
        fs.append(f.copy())
        xs.append(x.copy())
        for t in range(max(k - 1, 1), k + 1):
            axis = (t - 1) % 3
            g = f[axis].real
            expected = expected - g * (xs[t - 1] - xs[t] + 0.5 * (fs[t - 1] - fs[t]))
        assert np.max(np.abs(out - expected)) < 1e-12


def test_metric_zero_mode_and_high_g():
    """refscf.rs:160-171: weights zero at G = 0 and off the smooth sphere; 100 pi."""
    w = B.metric_weights(2.0, [0.0, 1.0, 4.0, 9.0], [True, True, True, False])
    a = np.array([900, 1 + 2j, 2 - 1j, 40])
    b = np.array([-500, 3 - 1j, -1 + 2j, 70])
    assert abs(B.metric_dot(w, a, b)) < 1e-13
    assert abs(B.metric_dot(w, a, a) - 100 * math.pi) < 1e-12


def test_thomas_fermi_is_opt_in_and_high_g_mixes_simply():
    """refscf.rs:172-195."""
    mix = B.Broyden([0.0, 1.0, 9.0], [True, True, False], 10.0, 2.0, MV, beta=0.7, thomas_fermi=True)
    out, _ = mix.update([2.0, 3.0, 4.0], [0.0, 1.0, 2.0])
    rs = (30.0 / (8.0 * math.pi)) ** (1 / 3)
    a = (12.0 / math.pi) ** (2 / 3) / rs
    assert out[0] == 2.0
    assert abs(out[1].real - (3.0 + 0.7 / (1.0 + a))) < 1e-14
    assert out[2] == 5.4


def test_singular_history_is_an_error():
    """refscf.rs:196-207."""
    mix = B.Broyden([1.0], [True], 1.0, 2.0, MV)
    mix.update([0.0], [1.0])
    with pytest.raises(B.Singular):
        mix.update([1.0], [1.0])
