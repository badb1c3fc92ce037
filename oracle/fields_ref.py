"""Oracle (test infrastructure only): numpy restatement of the SCF-map steps next to
the Hamiltonian apply.  Only tests/ import this module.

* band_density_sum: sum_b w_b |psi_b(r)|^2 / volume in band order, psi_b the unscaled
  inverse transform sum_G c_G e^{+iGr} of column b on the C-order grid
  (crates/dft-physics/src/distributed_complex.rs:485-547; Gamma ORC columns
  crates/dft-physics/src/distributed_real_gamma.rs:744-785, expanded to the full
  sphere with c_0 = x_0, c_{+G_i} = (x_{2i-1} + i x_{2i}) / sqrt 2, c_{-G} = conj c_G,
  crates/dft-basis/src/half.rs:31-37).
* lda_pz: Slater exchange and PZ81 correlation per point
  (crates/dft-physics/src/xc.rs:39-77), zero at or below 1e-10.
* fields: the field step of a map with LDA-PZ and no core density
  (crates/dft-engine/src/refscf/map.rs:41-198): rho(G) = FFT(rho)/N, V_H(G) =
  4 pi rho(G) / |G|^2 (G = 0 zero; canonical Miller index of every grid point,
  |G|^2 as crates/dft-engine/src/refscf/density.rs:17-26), V_H = Re IFFT*N;
  v_xc = LDA-PZ(|rho|); energies dV/2 sum rho V_H, dV sum |rho| eps_xc, dV sum rho v_xc.
* add_local_change: hx + FFT(dV(r) IFFT(x))/N on the sphere rows
  (crates/dft-physics/src/distributed_complex.rs:388-420).
"""
from __future__ import annotations

import numpy as np

DENSITY_THRESHOLD = 1e-10


def expand_orc(x, plus, minus):
    """Full-sphere complex coefficients (npw, m) of real ORC columns (npw, m)."""
    x = np.asarray(x, dtype=np.float64)
    c = np.zeros(x.shape, dtype=np.complex128)
    c[plus[0]] = x[0]
    i = np.arange(1, len(plus))
    v = (x[2 * i - 1] + 1j * x[2 * i]) / np.sqrt(2.0)
    c[plus[1:]] = v
    c[minus[1:]] = np.conj(v)
    return c


def to_real(dims, index, c):
    """Unscaled inverse transforms of the columns of c (npw, m): (m, n0, n1, n2)."""
    n = int(np.prod(dims))
    out = np.empty((c.shape[1],) + tuple(dims), dtype=np.complex128)
    for b in range(c.shape[1]):
        g = np.zeros(n, dtype=np.complex128)
        g[index] = c[:, b]
        out[b] = np.fft.ifftn(g.reshape(dims)) * n
    return out


def band_density_sum(dims, index, c, weights, volume):
    """c: complex sphere coefficients (npw, m) (Gamma: expand_orc first)."""
    psi = to_real(dims, index, c)
    rho = np.zeros(tuple(dims))
    for b, w in enumerate(weights):
        rho += w * (psi[b].real ** 2 + psi[b].imag ** 2) / volume
    return rho


def lda_pz(n):
    """(eps_xc, v_xc) per point of a non-negative density array."""
    n = np.asarray(n, dtype=np.float64)
    eps = np.zeros_like(n)
    v = np.zeros_like(n)
    m = n > DENSITY_THRESHOLD
    a = n[m]
    rs = np.cbrt(3.0 / (4.0 * np.pi)) / np.cbrt(a)
    eps_x = -0.75 * np.cbrt(3.0 / np.pi) * np.cbrt(a)
    hi = rs >= 1.0
    eps_c = np.empty_like(a)
    der = np.empty_like(a)
    r = rs[hi]
    den = 1.0 + 1.0529 * np.sqrt(r) + 0.3334 * r
    eps_c[hi] = -0.1423 / den
    der[hi] = 0.1423 * (1.0529 / (2.0 * np.sqrt(r)) + 0.3334) / den ** 2
    r = rs[~hi]
    eps_c[~hi] = 0.0311 * np.log(r) - 0.048 + 0.0020 * r * np.log(r) - 0.0116 * r
    der[~hi] = 0.0311 / r + 0.0020 * (np.log(r) + 1.0) - 0.0116
    eps[m] = eps_x + eps_c
    v[m] = 4.0 * eps_x / 3.0 + eps_c - rs * der / 3.0
    return eps, v


def squared_frequencies(rows, dims):
    """|G|^2 of every grid point's canonical Miller index (lattice vectors = rows)."""
    recip = 2.0 * np.pi * np.linalg.inv(np.asarray(rows, dtype=np.float64).reshape(3, 3)).T  # rows: b_j
    ms = []
    for n in dims:
        i = np.arange(n)
        ms.append(np.where(i <= (n - 1) // 2, i, i - n).astype(np.float64))
    m0, m1, m2 = np.meshgrid(*ms, indexing="ij")
    g = m0[..., None] * recip[0] + m1[..., None] * recip[1] + m2[..., None] * recip[2]
    return np.sum(g * g, axis=-1)


def fields(rows, density):
    """(v_hxc, v_h, hartree, xc, xc_integral) of a signed density grid."""
    rho = np.asarray(density, dtype=np.float64)
    dims = rho.shape
    n = rho.size
    volume = abs(np.linalg.det(np.asarray(rows, dtype=np.float64).reshape(3, 3)))
    dv = volume / n
    coeff = np.fft.fftn(rho) / n
    g2 = squared_frequencies(rows, dims)
    g2[0, 0, 0] = 1.0
    coeff = coeff * (4.0 * np.pi / g2)
    coeff[0, 0, 0] = 0.0
    vh = (np.fft.ifftn(coeff) * n).real
    eh = 0.5 * dv * np.sum(rho * vh)
    a = np.abs(rho)
    eps, vxc = lda_pz(a)
    ex = dv * np.sum(a * eps)
    vx = dv * np.sum(rho * vxc)
    return vh + vxc, vh, eh, ex, vx


def add_local_change(dims, index, c, change, hc):
    """hc + FFT(change * IFFT(c))/N on the sphere rows (complex coefficients)."""
    n = int(np.prod(dims))
    out = np.array(hc, dtype=np.complex128)
    psi = to_real(dims, index, c)
    for b in range(c.shape[1]):
        out[:, b] += np.fft.fftn(psi[b] * change).reshape(-1)[index] / n
    return out
