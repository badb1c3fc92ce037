"""Oracle (test infrastructure only): numpy restatement of the reference density mixer
and its metric.  Only tests/ import this module.

* Metric (crates/dft-engine/src/refscf/metric.rs:1-60, 147-200): the half-sphere
  Hartree form w_G Re(conj(a_G) b_G) with w_G = 8 pi Omega / G^2 for smooth G != 0 and
  0 otherwise (Ry), summed with Neumaier compensation.
* Broyden (crates/dft-engine/src/refscf/broyden.rs:96-123, 319-435): unnormalised
  difference-history Anderson update.  Iteration k stores dF = F_prev - F and
  dx = x_prev - x in ring slot (k-2) mod history (k = 1 only saves x, F); the Gram
  A_ij = <dF_i, dF_j> and b_i = <dF_i, F>; A = Q diag(lambda) Q^T, an error when
  lambda_min <= p eps lambda_max; gamma = Q diag(1/lambda) Q^T b; on smooth G
  x~ = x - gamma.dx, F~ = F - gamma.dF, next = x~ + beta s_G F~ with the Thomas-Fermi
  screening s_G = G^2/(G^2 + a) (a = (12/pi)^(2/3)/r_s) when enabled, else 1; other G
  mix simply (next = x + beta F).
"""
from __future__ import annotations

import math

import numpy as np

EPS = np.finfo(np.float64).eps


class Singular(ValueError):
    pass


def metric_weights(volume, g2, smooth):
    g2 = np.asarray(g2, dtype=np.float64)
    smooth = np.asarray(smooth, dtype=bool)
    w = np.zeros_like(g2)
    m = smooth & (g2 > 0)
    w[m] = 8.0 * math.pi * volume / g2[m]
    return w


def metric_dot(weights, a, b):
    """Neumaier-compensated sum of w Re(conj(a) b) in index order (metric.rs:175-190)."""
    v = weights * (np.real(a) * np.real(b) + np.imag(a) * np.imag(b))
    s, c = 0.0, 0.0
    for x in v.tolist():
        t = s + x
        c += (s - t) + x if abs(s) >= abs(x) else (x - t) + s
        s = t
    return s + c


class Broyden:
    def __init__(self, g2, smooth, volume, electrons, metric_volume, beta=0.7, history=8, thomas_fermi=False):
        if not (0.0 < beta <= 1.0) or not (1 <= history <= 25):
            raise ValueError("profile")
        g2 = np.asarray(g2, dtype=np.float64)
        self.smooth = np.asarray(smooth, dtype=bool)
        self.beta, self.history = beta, history
        rs = (3.0 * volume / (4.0 * math.pi * electrons)) ** (1.0 / 3.0)
        a = (12.0 / math.pi) ** (2.0 / 3.0) / rs
        self.screening = g2 / (g2 + a) if thomas_fermi else np.ones_like(g2)
        self.weights = metric_weights(metric_volume, g2, smooth)
        n = len(g2)
        self.iteration = 0
        self.prev_x = np.zeros(n, np.complex128)
        self.prev_f = np.zeros(n, np.complex128)
        self.df = np.zeros((history, n), np.complex128)
        self.dx = np.zeros((history, n), np.complex128)
        self.gamma = np.zeros(0)
        self.reduced = np.zeros(n, np.complex128)

    def occupancy(self):
        return min(max(self.iteration - 1, 0), self.history)

    def update(self, x, f):
        x = np.asarray(x, np.complex128)
        f = np.asarray(f, np.complex128)
        self.iteration += 1
        slot = (self.iteration - 2) % self.history if self.iteration > 1 else None
        p = self.occupancy()
        if slot is not None:
            self.df[slot] = self.prev_f - f
            self.dx[slot] = self.prev_x - x
        self.prev_x = x.copy()
        self.prev_f = f.copy()
        gamma = np.zeros(p)
        cond = None
        if p > 0:
            A = np.zeros((p, p))
            for i in range(p):
                for j in range(i + 1):
                    A[i, j] = A[j, i] = metric_dot(self.weights, self.df[i], self.df[j])
            b = np.array([metric_dot(self.weights, self.df[i], f) for i in range(p)])
            lam, Q = np.linalg.eigh(A)
            lo, hi = lam[0], lam[-1]
            cond = hi / lo if lo > 0 else math.inf
            if lo <= p * EPS * hi or not math.isfinite(cond):
                raise Singular(f"singular history at iteration {self.iteration}")
            for j in range(p):
                proj = float(Q[:, j] @ b)
                gamma += Q[:, j] * (proj / lam[j])
        self.gamma = gamma
        xx = x.copy()
        ff = f.copy()
        s = self.smooth
        if p > 0:
            xx[s] -= gamma @ self.dx[:p][:, s]
            ff[s] -= gamma @ self.df[:p][:, s]
        self.reduced = ff.copy()
        ff[s] *= self.screening[s]
        nxt = xx + self.beta * ff
        return nxt, {"iteration": self.iteration, "occupancy": p, "slot": slot, "condition": cond}
