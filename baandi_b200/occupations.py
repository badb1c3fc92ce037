"""Fermi-Dirac occupations of a spin-unpolarised k-point set (host; small arrays).

Restates crates/dft-physics/src/occupations.rs:57-235 for one channel of capacity 2:
the fraction p(x) = 1 / (1 + e^x) and entropy s(x) = ln(1 + e^-|x|) + |x| q (q the
smaller tail) from exp(-|x|) only; the chemical potential is bracketed by widening
[e_min - w, e_max + w] from w = theta, then located until the weighted count is within
1e-13 of the target; TS = theta sum_k w_k 2 s((e - mu) / theta).  The reference bisects;
here each step takes the Newton step on the count (slope sum_k w_k 2 p (1 - p) / theta)
when it falls inside the bracket and the midpoint otherwise, so the same stopping rule is
met in a few steps instead of about forty.
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

    ef = e.ravel()
    wf = np.broadcast_to((2.0 * w)[:, None], e.shape).ravel()

    def fractions(mu):
        x = (ef - mu) / theta_ha
        t = np.exp(-np.abs(x))
        return np.where(x >= 0.0, t, 1.0) / (1.0 + t), t

    def number(mu):
        return float(wf @ fractions(mu)[0])

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
    x = 0.5 * lo + 0.5 * hi
    for _ in range(max_iterations):
        p, t = fractions(x)
        count = float(wf @ p)
        if abs(count - electrons) <= tolerance * electrons:
            mu = x
            break
        if count < electrons:
            lo = x
        else:
            hi = x
        slope = float(wf @ (t / (1.0 + t) ** 2)) / theta_ha
        nxt = x - (count - electrons) / slope if slope > 0.0 else lo - 1.0
        if not (lo < nxt < hi):
            nxt = 0.5 * lo + 0.5 * hi
            if nxt in (lo, hi):
                break
        x = nxt
    if mu is None:
        raise ValueError("the electron count did not converge")
    p, s = _fraction_entropy((e - mu) / theta_ha)
    occ = [2.0 * row for row in p]
    ts = theta_ha * float(np.sum(w[:, None] * 2.0 * s))
    return occ, mu, ts
