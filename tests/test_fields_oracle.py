"""Pins of the field-step oracle (Hartree, LDA-PZ, band density) against the
reference's own known-answer tests (CPU only).  Each test names the reference test it
restates."""
import math

import numpy as np

from oracle import fields_ref as F

A_SI = 5.43 / 0.529177210903  # 5.43 Angstrom in Bohr, the reference fixtures' Si cell
SI_ROWS = np.array([[0, A_SI / 2, A_SI / 2], [A_SI / 2, 0, A_SI / 2], [A_SI / 2, A_SI / 2, 0]])


def _rel(a, b):
    return abs(a - b) / abs(b)


def test_hartree_analytic_cosine():
    """crates/dft-physics/src/tests.rs:80-150 (hartree_analytic): uniform density gives
    zero potential and energy; 0.3 + 2A cos(2 pi (i/n0 - j/n1)) gives
    E_H = 4 pi V A^2 / |G|^2 and V_H = 8 pi A / |G|^2 cos, both to 1e-12; linearity."""
    dims = (12, 10, 9)
    vol = abs(np.linalg.det(SI_ROWS))
    _, vh0, e0, _, _ = F.fields(SI_ROWS, np.full(dims, 0.3))
    assert abs(e0) < 1e-14 and np.max(np.abs(vh0)) < 1e-14
    amp = 0.02
    i, j, _ = np.meshgrid(*(np.arange(n) for n in dims), indexing="ij")
    cosine = np.cos(2 * np.pi * (i / dims[0] - j / dims[1]))
    n = 0.3 + 2 * amp * cosine
    _, vh, eh, _, _ = F.fields(SI_ROWS, n)
    g2 = F.squared_frequencies(SI_ROWS, dims)[1, dims[1] - 1, 0]
    assert _rel(eh, 4 * math.pi * vol * amp * amp / g2) < 1e-12
    vscale = 8 * math.pi * amp / g2
    assert np.max(np.abs(vh - vscale * cosine)) / vscale < 1e-12
    second = 0.1 + 0.01 * np.cos(2 * np.pi * (j / 10 + np.arange(9)[None, None, :] / 9))
    _, vh2, _, _, _ = F.fields(SI_ROWS, second)
    _, vhc, _, _, _ = F.fields(SI_ROWS, 0.7 * n + 1.3 * second)
    assert np.max(np.abs(vhc - 0.7 * vh - 1.3 * vh2)) / vscale < 1e-12


def test_hartree_nyquist_and_odd_grids():
    """crates/dft-physics/src/tests.rs:381-430: on the skew Si cell the two Fourier
    components of 0.2 + 0.02 cos(2 pi (-3 i/n0 + j/5)) have their own |G|^2 (a
    negative even Nyquist index on 6 points); E_H = sum 1/2 V 4 pi 0.01^2 / |G|^2."""
    vol = abs(np.linalg.det(SI_ROWS))
    recip = 2 * np.pi * np.linalg.inv(SI_ROWS).T
    for dims, millers in (((6, 5, 7), ((-3, 1, 0), (-3, -1, 0))), ((7, 5, 7), ((-3, 1, 0), (3, -1, 0)))):
        i, j, _ = np.meshgrid(*(np.arange(n) for n in dims), indexing="ij")
        n = 0.2 + 0.02 * np.cos(2 * np.pi * (-3 * i / dims[0] + j / 5))
        _, _, eh, _, _ = F.fields(SI_ROWS, n)
        expected = 0.0
        for m in millers:
            g = np.asarray(m, float) @ recip
            expected += 0.5 * vol * 4 * math.pi * 0.01 ** 2 / float(g @ g)
        assert _rel(eh, expected) < 1e-12


def test_lda_pz_cross_checks():
    """crates/dft-physics/src/tests.rs:152-216 (xc_cross_checks): Slater exchange in
    closed form and v_x = 4/3 eps_x to 1e-12; v_xc the derivative of n eps_xc
    (central difference, 1e-7); the PZ81 jump at rs = 1 to 1e-10; a uniform grid's
    E_xc and integral n v_xc to 1e-12."""
    n = 10.0 ** (-6 + np.arange(71) / 10)
    eps, v = F.lda_pz(n)
    closed = -3 / (4 * np.pi) * np.cbrt(3 * np.pi ** 2 * n)
    rs = np.cbrt(3 / (4 * np.pi)) / np.cbrt(n)
    hi = rs >= 1
    den = 1 + 1.0529 * np.sqrt(rs) + 0.3334 * rs
    ec = np.where(hi, -0.1423 / den, 0.0311 * np.log(rs) - 0.048 + 0.002 * rs * np.log(rs) - 0.0116 * rs)
    assert np.max(np.abs(eps - ec - closed) / np.abs(closed)) < 1e-12
    for r in list(0.1 * 200.0 ** (np.arange(101) / 100)) + [0.999, 1.001]:
        d = 3 / (4 * np.pi * r ** 3)
        h = d * 1e-5
        fd = ((d + h) * F.lda_pz(np.array([d + h]))[0][0] - (d - h) * F.lda_pz(np.array([d - h]))[0][0]) / (2 * h)
        vv = F.lda_pz(np.array([d]))[1][0]
        assert abs(vv - fd) / abs(fd) < 1e-7
    left = 3 / (4 * np.pi * (1 - 1e-10) ** 3)
    right = 3 / (4 * np.pi * (1 + 1e-10) ** 3)
    (el, er), (vl, vr) = F.lda_pz(np.array([left, right]))
    ex_l = -0.75 * np.cbrt(3 / np.pi) * np.cbrt(left)
    ex_r = -0.75 * np.cbrt(3 / np.pi) * np.cbrt(right)
    jump_eps = -0.1423 / (1 + 1.0529 + 0.3334) - (-0.048 - 0.0116)
    jump_v = (-0.1423 / (1 + 1.0529 + 0.3334) - 0.1423 * (1.0529 / 2 + 0.3334) / (3 * (1 + 1.0529 + 0.3334) ** 2)
              - (-0.048 - 0.0116 - (0.0311 + 0.0020 - 0.0116) / 3))
    assert abs((er - ex_r) - (el - ex_l) - jump_eps) < 1e-10
    assert abs((vr - 4 * ex_r / 3) - (vl - 4 * ex_l / 3) - jump_v) < 1e-10
    a = 270.0 ** (1 / 3)
    rho = np.full((4, 5, 6), 0.1)
    _, _, _, ex, vx = F.fields(np.diag([a, a, a]), rho)
    e1, v1 = F.lda_pz(np.array([0.1]))
    assert _rel(ex, 270 * 0.1 * e1[0]) < 1e-12
    assert _rel(vx, 270 * 0.1 * v1[0]) < 1e-12


def test_lda_pz_thresholds():
    """crates/dft-physics/src/tests.rs:219-232 (validation_and_thresholds): zero at or
    below 1e-10, negative just above; the map evaluates LDA on |rho| so signed input
    only flips the sign of the density factor (crates/dft-engine/src/refscf/map.rs:
    124-163)."""
    eps, v = F.lda_pz(np.array([0.0, 1e-12, 1e-10]))
    assert np.all(eps == 0) and np.all(v == 0)
    assert F.lda_pz(np.array([1.00001e-10]))[0][0] < 0
    rho = np.full((3, 4, 5), -0.05)
    hxc, vh, _, ex, vx = F.fields(np.diag([6.0, 6.0, 6.0]), rho)
    e1, v1 = F.lda_pz(np.array([0.05]))
    vol = 216.0
    assert _rel(ex, vol * 0.05 * e1[0]) < 1e-12
    assert _rel(vx, -vol * 0.05 * v1[0]) < 1e-12
    assert np.max(np.abs(hxc - vh - v1[0])) < 1e-15


def test_band_density_normalisation():
    """distributed_complex.rs:485-547: a normalised band of weight w carries w electrons:
    dV sum_r w |psi|^2 / volume = w (Parseval with the unscaled inverse transform), and
    a Gamma ORC column expands to a real function."""
    rng = np.random.default_rng(5)
    dims = (8, 9, 10)
    n = int(np.prod(dims))
    idx = rng.choice(n, 40, replace=False)
    c = rng.standard_normal((40, 3)) + 1j * rng.standard_normal((40, 3))
    c /= np.linalg.norm(c, axis=0)
    w = np.array([2.0, 0.5, 0.0])
    vol = 123.0
    rho = F.band_density_sum(dims, idx, c, w, vol)
    assert abs(rho.sum() * vol / n - w.sum()) < 1e-12
    plus = np.array([0, 1, 3])
    minus = np.array([0, 2, 4])
    x = rng.standard_normal((5, 2))
    cc = F.expand_orc(x, plus, minus)
    flat = lambda m: int(np.ravel_multi_index(tuple(np.mod(m, dims)), dims))
    sphere = [flat((0, 0, 0)), flat((0, 0, 1)), flat((0, 0, -1)), flat((1, 2, 3)), flat((-1, -2, -3))]
    psi = F.to_real(dims, np.array(sphere), cc)
    assert np.max(np.abs(psi.imag)) < 1e-12
