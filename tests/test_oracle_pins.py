"""Pins of the oracle against the reference's own test recipes and known answers
(CPU only).  Each test names the reference test it restates."""
import math

import numpy as np
import pytest

from oracle import davidson_ref as D
from oracle import oracle as O
from oracle import setup_ref as S

A_SI = 5.43 / 0.529177210903  # 5.43 Angstrom in Bohr (CODATA 2018), the reference fixtures' cell


def _fcc(a):
    return S.Cell(np.array([[0, a / 2, a / 2], [a / 2, 0, a / 2], [a / 2, a / 2, 0]]))


def _dense_setup():
    """crates/dft-physics/tests/all/hamiltonian.rs:20-31 and :289-330."""
    cell = _fcc(A_SI)
    b = S.basis_at_k(cell, 3.0)
    ps = S.reference_test_pseudo(801)
    pos = np.array([[0, 0, 0], [A_SI / 4] * 3])
    sp = [S.Species(ps, pos)]
    nl = S.nonlocal_table(b, cell.volume, sp)
    dims, _ = S.grid_dims(cell, 3.0)
    dens = S.basis_at_k(cell, 12.0)
    coeff = {(0, 0, 0): 0.17 + 0j, (1, 0, 0): 0.07 + 0.03j, (-1, 0, 0): 0.07 - 0.03j,
             (0, 1, -1): -0.04 + 0.02j, (0, -1, 1): -0.04 - 0.02j}
    for m, v in zip(dens.miller.tolist(), S.ionic_local(dens, cell.volume, sp)):
        coeff[tuple(m)] = coeff.get(tuple(m), 0) + v
    v = O.sampled_potential(dims, coeff)
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    return cell, b, nl, dims, coeff, v, idx


def _random(n, seed):
    """LCG of the reference fixture (hamiltonian.rs:32-38)."""
    out = []
    s = seed
    for _ in range(2 * n):
        s = (s * 6364136223846793005 + 1) % (1 << 64)
        out.append((s >> 11) / float(1 << 53) - 0.5)
    a = np.array(out)
    return a[0::2] + 1j * a[1::2]


def test_dense_hamiltonian_equalities():
    """hamiltonian.rs:289-417: convolution < 1e-12, entries < 1e-11, Hermiticity < 1e-12,
    block = single < 1e-14, constant potential < 1e-12, free-electron spectrum < 1e-12."""
    cell, b, nl, dims, coeff, v, idx = _dense_setup()
    n = b.npw
    H = O.dense_hamiltonian(b, coeff, nl)
    Hloc = O.dense_hamiltonian(b, coeff, None)
    empty = S.Nonlocal(np.zeros((n, 0), np.complex128), [], [])
    x, y = _random(n, 18), _random(n, 46)
    kin = 0.5 * b.kpg2
    loc = O.apply_complex(dims, idx, v, kin, empty, x[:, None])[:, 0]
    assert np.max(np.abs(loc - Hloc @ x)) < 1e-12
    eye = np.eye(n, dtype=np.complex128)
    cols = O.apply_complex(dims, idx, v, kin, nl, eye)
    assert np.max(np.abs(cols - H)) < 1e-11
    ax = O.apply_complex(dims, idx, v, kin, nl, x[:, None])[:, 0]
    ay = O.apply_complex(dims, idx, v, kin, nl, y[:, None])[:, 0]
    herm = abs(np.vdot(x, ay) - np.vdot(ax, y)) / max(abs(np.vdot(x, ay)), abs(np.vdot(ax, y)))
    assert herm < 1e-12
    block = O.apply_complex(dims, idx, v, kin, nl, np.stack([x, y], axis=1))
    assert max(np.max(np.abs(block[:, 0] - ax)), np.max(np.abs(block[:, 1] - ay))) < 1e-14
    const = O.apply_complex(dims, idx, np.full(dims, 0.23), kin, empty, x[:, None])[:, 0]
    assert np.max(np.abs(const - x * (kin + 0.23))) < 1e-12
    hc = O.apply_complex(dims, idx, np.full(dims, 0.23), kin, empty, eye)
    free = np.linalg.eigvalsh(0.5 * (hc + hc.conj().T))
    assert np.max(np.abs(free - np.sort(kin + 0.23))) < 1e-12


def test_fft_conventions_signed_modes():
    """docs/physics-conventions.md:61-78, 115-124 of the reference: to_real is unscaled
    exp(+iGr), to_reciprocal scales 1/N; signed modes (1,-1,2) -> index (1,4,2) and
    (-2,1,-3) -> (2,1,3) on 4x5x6; round trip < 1e-12; Parseval."""
    dims = (4, 5, 6)
    for miller, index in [((1, -1, 2), (1, 4, 2)), ((-2, 1, -3), (2, 1, 3))]:
        g = np.zeros(dims, np.complex128)
        g[index] = 1.0
        f = O.fft3d(g, +1)
        i, j, k = np.meshgrid(*[np.arange(d) / d for d in dims], indexing="ij")
        expect = np.exp(2j * math.pi * (miller[0] * i + miller[1] * j + miller[2] * k))
        assert np.max(np.abs(f - expect)) < 1e-12
        back = O.fft3d(f, -1)
        assert np.max(np.abs(back - g)) < 1e-12
    rng = np.random.default_rng(3)
    for shape in [(4, 5, 6), (15, 20, 24), (16, 16, 16), (27, 27, 27)]:
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        r = O.fft3d(a, +1)
        assert np.max(np.abs(O.fft3d(r, -1) - a)) / np.max(np.abs(a)) < 1e-12
        n = np.prod(shape)
        assert abs(np.sum(np.abs(r) ** 2) / n - np.sum(np.abs(a) ** 2)) / np.sum(np.abs(a) ** 2) < 1e-12


def test_gamma_pair_path_equals_complex_path():
    """The real ORC apply (distributed_real_gamma.rs:1062-1352) is the complex apply on
    Hermitian vectors in orthonormal real coordinates."""
    cell, b, nl, dims, coeff, v, idx = _dense_setup()
    plus, minus, _ = S.half_sphere(b)
    rng = np.random.default_rng(5)
    xr = rng.standard_normal((b.npw, 5))
    yr = O.apply_gamma(dims, idx, plus, minus, v, S.orc_kinetic(plus, b.kpg2), S.orc_projectors(plus, nl.table), nl,
                       xr)
    for c in range(5):
        full = S.orc_unpack(plus, minus, xr[:, c])
        hf = O.apply_complex(dims, idx, v, 0.5 * b.kpg2, nl, full[:, None])[:, 0]
        assert np.max(np.abs(S.orc_pack(plus, minus, hf) - yr[:, c])) < 1e-12


def test_half_sphere_four_shapes():
    """crates/dft-basis/src/half.rs:190-232 (mirrors_and_orc_four_shapes)."""
    for rows in ([[8., 0., 0.], [0., 8., 0.], [0., 0., 8.]], [[8., 1., 0.], [0., 7., 2.], [1., 0., 9.]],
                 [[4., 0., 0.], [0., 5., 0.], [0., 0., 20.]], [[7., 0., 0.], [0., 8., 0.], [0., 0., 25.]]):
        cell = S.Cell(np.array(rows))
        b = S.basis_at_k(cell, 1.0)
        plus, minus, mirror = S.half_sphere(b)
        n = b.npw
        assert 2 * len(plus) - 1 == n
        assert np.all(mirror[mirror] == np.arange(n))
        assert np.all(np.diff(plus[1:]) > 0)
        x = np.array([math.sin(i * 17 + 3) for i in range(n)]) / math.sqrt(n)
        y = np.array([math.cos(i * 7 + 1) for i in range(n)]) / math.sqrt(n)
        a, c = S.orc_unpack(plus, minus, x), S.orc_unpack(plus, minus, y)
        dot, cdot = x @ y, np.vdot(a, c)
        defect = max(abs(dot - cdot.real), abs(cdot.imag), abs(x @ x - np.vdot(a, a).real))
        assert defect < 1e-15
        assert np.max(np.abs(S.orc_pack(plus, minus, a) - x)) < 1e-15


def test_grid_and_kmesh_rules():
    """crates/dft-basis/src/lib.rs:414-455 (2,3,5-smooth round-up) and
    crates/dft-geometry/src/kpoints.rs:63-116 (4x4x4 unshifted mesh, 36 TR classes)."""
    dims, req = S.grid_dims(_fcc(10.26), 15.0)
    assert req == [25, 25, 25] and dims == [25, 25, 25]
    dims, req = S.grid_dims(S.Cell(np.diag([10.26] * 3)), 20.0)
    assert req == [41, 41, 41] and dims == [45, 45, 45]
    ks = S.reduce_time_reversal(S.monkhorst_pack((4, 4, 4)))
    assert len(ks) == 36 and abs(sum(w for _, w in ks) - 1.0) < 1e-14
    assert len(S.reduce_time_reversal(S.monkhorst_pack((2, 2, 2)))) == 8
    with pytest.raises(ValueError):
        S.grid_dims(_fcc(10.26), 15.0, override=[24, 24, 24])


@pytest.mark.parametrize("cluster", [False, True])
def test_davidson_oracle_dense_fixture(cluster):
    """crates/dft-solvers/tests/ref_davidson.rs:113-228: sorted roots within 1e-11 of the
    dense eigensolver and occupied projectors within 2e-6, all bands converged."""
    dim, bands, occupied = 32, 8, 6
    h = D.dct_fixture(dim, cluster)
    exact, q = np.linalg.eigh(h)
    opts = D.Options(bands, 1e-13, occupied, first_step=True, max_iterations=400)
    sol = D.solve(lambda x: h @ x, D.dct_start(dim, bands), np.diag(h).copy(), opts)
    assert sol.converged.all()
    assert np.max(np.abs(sol.eigenvalues - exact[:bands])) < 1e-11
    assert D.projector_error(sol.eigenvectors, q, occupied) < 2e-6
    assert sol.contractions > 0


def test_band_thresholds_and_denominator():
    """ref_davidson.rs tests thresholds_preconditioner_and_invalid_input (:231-258)."""
    o = D.Options(4, 2e-8, 2)
    assert o.band_threshold(0) == 2e-8 and o.band_threshold(3) == 5e-6
    o.first_step = True
    assert o.band_threshold(3) == 2e-8
    for d in [-1e8, -10.0, -1.0, 0.0, 0.5, 1.0, 100.0]:
        p = float(D.preconditioner_denominator(d, 0.0))
        direct = 0.25 * (1.0 + 2.0 * d + math.sqrt(1.0 + (2.0 * d - 1.0) ** 2))
        assert math.isfinite(p) and p > 0 and abs(p - direct) < 1e-8
    for h, e in [(-0.7, -0.2), (0.35, -0.15), (2.1, 0.6)]:
        x = 2.0 * (h - e)
        d_ry = (1.0 + x + math.sqrt(1.0 + (x - 1.0) ** 2)) / 2.0
        assert abs(2.0 * float(D.preconditioner_denominator(h, e)) - d_ry) < 2e-15
        assert abs(float(D.preconditioner_denominator(h, e)) - float(D.preconditioner_denominator(h + .25, e + .25))) \
            < 2e-15


def test_tpa_and_ritz_shift_corrections():
    """crates/dft-solvers/tests/all/preconditioner_variants.rs:9-37: TPA uses the
    selected band's kinetic expectation with the 0.1 Ha floor (-1 at t = 0, -65/81 at
    t = s, finite and negative at t = 1e200); Ritz shift floors h - lambda at 0.1."""
    d = np.array([0.0, 0.1, 0.2, 1e200])
    r = np.ones(4)
    v0 = np.array([0.0, 0.0, 2.0, 0.0])
    y = D.correction("tpa", r, v0, d, 0.0)
    assert y[0] == -1.0
    assert abs(y[2] + 65.0 / 81.0) < 1e-15
    assert y[3] < 0 and np.isfinite(y[3])
    y = D.correction("tpa", r, np.array([1.0, 0, 0, 0]), d, 0.0)
    assert abs(y[1] + 65.0 / 81.0) < 1e-15
    y = D.correction("ritz_shift", r, v0, d, 0.2)
    assert np.all(y[:3] == -10.0) and y[3] < 0
