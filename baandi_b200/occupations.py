"""Fermi-Dirac occupations of a spin-unpolarised k-point set (host; small arrays).

Restates crates/dft-physics/src/occupations.rs:57-235 for one channel of capacity 2:
the fraction p(x) = 1 / (1 + e^x) and entropy s(x) = ln(1 + e^-|x|) + |x| q (q the
smaller tail) from exp(-|x|) only; the chemical potential is bracketed by widening
[e_min - w, e_max + w] from w = theta, then bisected until the weighted count is within
1e-13 of the target; TS = theta sum_k w_k 2 s((e - mu) / theta).
"""
from __future__ import annotations

import math

import numpy as np


def _fraction_entropy(x):
    a = np.abs(x)
    t = np.exp(-a)
    q = t / (1.0 + t)
    p = np.where(x >= 0.0, q, 1.0 / (1.0 + t))
    s = np.log1p(t) + np.where(np.isinf(a), 0.0, a * q)
    return p, s


def fermi_dirac(energies, weights, electrons: float, theta_ha: float, tolerance=1e-13, max_iterations=256):
    """energies: one ascending eigenvalue array per k point; weights: k weights
    (summing to one).  Returns (occupations per k (0..2), mu_ha, entropy_term_ha)."""
    e = np.stack([np.asarray(x, dtype=np.float64) for x in energies])
    w = np.asarray(weights, dtype=np.float64)
    if not (theta_ha > 0.0 and math.isfinite(theta_ha)):
        raise ValueError("smearing needs a positive finite theta in Ha")
    if not (0.0 < electrons < 2.0 * e.shape[1] * w.sum()):
        raise ValueError("no finite chemical potential for this electron count")

    def number(mu):
        p, _ = _fraction_entropy((e - mu) / theta_ha)
        return float(np.sum(w[:, None] * 2.0 * p))

    lo_e, hi_e = float(e.min()), float(e.max())
    width = theta_ha
    for _ in range(max_iterations):
        lo, hi = lo_e - width, hi_e + width
        if number(lo) <= electrons <= number(hi):
            break
        width *= 2.0
    else:
        raise ValueError("unable to bracket the chemical potential")
    mu = None
    for _ in range(max_iterations):
        mid = 0.5 * lo + 0.5 * hi
        count = number(mid)
        if abs(count - electrons) <= tolerance * electrons:
            mu = mid
            break
        if mid in (lo, hi):
            break
        if count < electrons:
            lo = mid
        else:
            hi = mid
    if mu is None:
        raise ValueError("the electron count did not converge")
    p, s = _fraction_entropy((e - mu) / theta_ha)
    occ = [2.0 * row for row in p]
    ts = theta_ha * float(np.sum(w[:, None] * 2.0 * s))
    return occ, mu, ts
