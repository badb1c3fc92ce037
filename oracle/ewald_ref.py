"""Oracle (test infrastructure only): the Ewald energy of point charges in a
neutralising background, restated from the standard Ewald split (the reference's
crates/dft-physics/src/ewald.rs computes the same energy), with a free splitting
parameter eta so that tests can check the eta independence.  Only tests/ import this
module."""
from __future__ import annotations

import itertools
import math

import numpy as np


def energy(rows, positions, charges, eta=None, t=7.0):
    a = np.asarray(rows, dtype=np.float64).reshape(3, 3)        # rows: lattice vectors
    b = 2.0 * math.pi * np.linalg.inv(a).T                      # rows: reciprocal vectors
    omega = abs(np.linalg.det(a))
    eta = math.sqrt(math.pi) / omega ** (1.0 / 3.0) if eta is None else eta
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    z = np.asarray(charges, dtype=np.float64)
    r_cut = t / eta + np.sum(np.linalg.norm(a, axis=1))
    g_cut = 2.0 * eta * t + np.sum(np.linalg.norm(b, axis=1))
    nr = [int(math.ceil(r_cut * np.linalg.norm(b[j]) / (2 * math.pi))) + 1 for j in range(3)]
    ng = [int(math.ceil(g_cut * np.linalg.norm(a[j]) / (2 * math.pi))) + 1 for j in range(3)]
    n = np.array(list(itertools.product(*(range(-m, m + 1) for m in nr))), dtype=np.float64)
    lat = n @ a
    real = 0.0
    for i in range(len(z)):
        d = pos[None, :, :] - pos[i][None, None, :] + lat[:, None, :]
        r = np.linalg.norm(d, axis=2)
        mask = (r > 0) & (r <= r_cut)
        vals = np.zeros_like(r)
        vals[mask] = np.array([math.erfc(eta * x) for x in r[mask]]) / r[mask]
        real += 0.5 * z[i] * np.sum(vals * z[None, :])
    m = np.array([v for v in itertools.product(*(range(-q, q + 1) for q in ng)) if any(v)], dtype=np.float64)
    g = m @ b
    g2 = np.sum(g * g, axis=1)
    keep = g2 <= g_cut * g_cut
    g, g2 = g[keep], g2[keep]
    s = np.exp(1j * (g @ pos.T)) @ z
    recip = 2.0 * math.pi / omega * np.sum(np.exp(-g2 / (4 * eta * eta)) / g2 * np.abs(s) ** 2)
    return real + recip - eta / math.sqrt(math.pi) * np.sum(z * z) - math.pi * np.sum(z) ** 2 / (2 * eta * eta * omega)
