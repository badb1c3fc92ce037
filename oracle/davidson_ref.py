"""Oracle (test infrastructure only): numpy restatement of the reference block
Davidson, crates/dft-solvers/src/ref_davidson.rs:117-366 (real Gamma ORC rows) and
crates/dft-solvers/src/ref_davidson_complex.rs:641-1110 (complex k points), one rank.

Setup V = start, HV = H V, S = V^H V, Cholesky with the pivot rule of
crates/dft-solvers/src/lean_davidson.rs:62-70 (squared pivot over the overlap
diagonal >= eps/1e-12), H_r = V^H H V, reduced eigenproblem.  Iterations: contraction
to the n Ritz vectors when m + active > capacity; corrections (HX - lambda X)/d with
the smooth denominator of ref_davidson.rs:418-422; drop |E| <= 32 eps; append, border,
bordered Cholesky, repair on a rejected pivot; H E; eigensolve; Ritz-change test with
the band thresholds of ref_davidson.rs:70-76.  The reduced eigensolves use numpy's
LAPACK; the reference uses faer (rounding-level differences only).

Only tests/ import this module.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

EPS = np.finfo(np.float64).eps
PIVOT_RATIO_MIN = EPS / 1e-12
DEPENDENCE_TOLERANCE = 1e-12


def preconditioner_denominator(h, e):
    """ref_davidson.rs:418-422 (Ry convention d_Ry = (1 + x + sqrt(1 + (x-1)^2))/2, x = 2(h-e))."""
    x = 2.0 * (np.asarray(h) - e)
    z = np.abs(x - 1.0)
    return 0.25 * (np.where(x >= 1.0, 2.0 * x, 2.0) + 1.0 / (np.hypot(z, 1.0) + z))


def tpa_weight(kinetic, scale):
    """crates/dft-solvers/src/lib.rs:194-206 (reciprocal form above the scale)."""
    t = np.asarray(kinetic, dtype=np.float64)
    x = t / scale
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        p_lo = 27.0 + x * (18.0 + x * (12.0 + x * 8.0))
        lo = p_lo / (p_lo + 16.0 * x ** 4)
        y = scale / t
        p_hi = y * (8.0 + y * (12.0 + y * (18.0 + y * 27.0)))
        hi = p_hi / (p_hi + 16.0)
    return np.where(x <= 1.0, lo, hi)


def kinetic_scale(weights, kinetic):
    """Weighted mean kinetic energy with the 0.1 Ha floor (lib.rs:176-192)."""
    w = np.asarray(weights, dtype=np.float64)
    return max(float(np.sum(w * kinetic) / np.sum(w)), 0.1)


def correction(kind, residual, x, diagonal, e):
    """One band's correction from its residual (the solver's preconditioner seam):
    'smooth' r / d(h, e) (ref_davidson.rs:418-422), 'tpa' -r tpa(t, s) with s the
    band's kinetic scale (lib.rs:240-277), 'ritz_shift' -r / max(h - e, 0.1)
    (lib.rs:300-309)."""
    d = np.asarray(diagonal)
    if kind == "tpa":
        return -residual * tpa_weight(d, kinetic_scale(np.abs(x) ** 2, d))
    if kind == "ritz_shift":
        return -residual / np.maximum(d - e, 0.1)
    return residual / preconditioner_denominator(d, e)


@dataclass
class Options:
    bands: int
    threshold: float
    occupied: int
    first_step: bool = False
    capacity: int = 0
    max_iterations: int = 20
    preconditioner: str = "smooth"

    def band_threshold(self, band: int) -> float:
        if self.first_step or band < self.occupied:
            return self.threshold
        return max(5.0 * self.threshold, 5e-6)


@dataclass
class Solution:
    eigenvalues: np.ndarray
    eigenvectors: np.ndarray
    converged: np.ndarray
    iterations: int = 0
    h_columns: int = 0
    hx: np.ndarray | None = None   # H applied to the eigenvectors
    repairs: int = 0
    contractions: int = 0
    ritz_changes: list = field(default_factory=list)


def _chol_extend(S, L, m0, m):
    for j in range(m0, m):
        for k in range(j):
            L[j, k] = (S[j, k] - np.dot(L[j, :k], np.conj(L[k, :k]))) / L[k, k].real
        d = S[j, j].real - np.sum(np.abs(L[j, :j]) ** 2)
        ratio = d / S[j, j].real
        if not (ratio >= PIVOT_RATIO_MIN) or not np.isfinite(ratio):
            return False
        L[j, j] = math.sqrt(d)
        L[:j, j] = 0.0
    return True


def _eigen(Hr, L, m):
    Lm = L[:m, :m]
    A = np.linalg.solve(Lm, Hr[:m, :m])
    A = np.linalg.solve(Lm, A.conj().T).conj().T
    A = 0.5 * (A + A.conj().T)
    w, Y = np.linalg.eigh(A)
    C = np.linalg.solve(Lm.conj().T, Y)
    return w, C


def solve(apply, start, diagonal, opts: Options, start_hx=None) -> Solution:
    """apply(X) -> H X for a (rows, k) block; start (rows, n); diagonal (rows,).  start_hx:
    H applied to the start block (the kept-HX start of
    crates/dft-solvers/src/ref_davidson_complex.rs:641 solve_with_initial_hx), else it is
    applied here.  The solution carries hx = H X of its eigenvectors (HV C)."""
    X0 = np.array(start)
    rows, n = X0.shape
    dt = X0.dtype
    cap = min(opts.capacity or 2 * n, rows)
    if n == 0 or n > rows or cap < min(2 * n, rows) or opts.occupied > n or opts.max_iterations == 0:
        raise ValueError("reference Davidson dimensions/threshold/start")
    V = np.zeros((rows, cap), dt)
    HV = np.zeros((rows, cap), dt)
    V[:, :n] = X0
    if start_hx is None:
        HV[:, :n] = apply(X0)
        sol = Solution(None, None, None, h_columns=n)
    else:
        HV[:, :n] = np.asarray(start_hx)
        sol = Solution(None, None, None, h_columns=0)
    S = np.zeros((cap, cap), dt)
    Hr = np.zeros((cap, cap), dt)
    L = np.zeros((cap, cap), dt)
    S[:n, :n] = V[:, :n].conj().T @ V[:, :n]
    if not _chol_extend(S, L, 0, n):
        raise ValueError("reference Davidson start is numerically dependent")
    Hr[:n, :n] = V[:, :n].conj().T @ HV[:, :n]
    w, C = _eigen(Hr, L, n)
    m = n
    active = list(range(n))
    conv = np.zeros(n, bool)

    def refresh(mm):
        nonlocal w, C
        S[:mm, :mm] = V[:, :mm].conj().T @ V[:, :mm]
        Hr[:mm, :mm] = V[:, :mm].conj().T @ HV[:, :mm]
        if not _chol_extend(S, L, 0, mm):
            raise ValueError("reference contracted basis is dependent")
        w, C = _eigen(Hr, L, mm)

    def contract(mm):
        nonlocal m
        sol.contractions += 1
        Vn = V[:, :mm] @ C[:, :n]
        HVn = HV[:, :mm] @ C[:, :n]
        V[:, :n] = Vn
        HV[:, :n] = HVn
        m = n
        refresh(n)

    for step in range(opts.max_iterations):
        if m + len(active) > cap and m > n:
            contract(m)
        if m + len(active) > cap and cap < rows:
            raise ValueError("capacity cannot hold the active correction block")
        Cs = C[:, active]
        Xs = V[:, :m] @ Cs
        HXs = HV[:, :m] @ Cs
        lam = w[active]
        E = np.stack([correction(opts.preconditioner, HXs[:, j] - Xs[:, j] * lam[j], Xs[:, j], diagonal, lam[j])
                      for j in range(len(active))], axis=1)
        norms = np.sqrt(np.sum(np.abs(E) ** 2, axis=0))
        if not np.all(np.isfinite(norms)):
            raise ValueError("nonfinite reference correction")
        keep = norms > 32.0 * EPS
        E = E[:, keep] / norms[keep][None, :]
        k = E.shape[1]
        need_repair = m + k > cap or k == 0
        if not need_repair:
            V[:, m:m + k] = E
            S[:m + k, m:m + k] = V[:, :m + k].conj().T @ E
            S[m:m + k, :m + k] = S[:m + k, m:m + k].conj().T
            if not _chol_extend(S, L, m, m + k):
                need_repair = True
        if need_repair:
            sol.repairs += 1
            Q = V[:, :m] @ C[:, :m]
            HQ = HV[:, :m] @ C[:, :m]
            V[:, :m], HV[:, :m] = Q, HQ
            S[:m, :m] = np.eye(m)
            L[:m, :m] = np.eye(m)
            Hr[:m, :m] = np.diag(w[:m])
            C = np.eye(m, dtype=dt)
            for _ in range(2):
                E = E - V[:, :m] @ (V[:, :m].conj().T @ E)
            cols = []
            for j in range(E.shape[1]):
                e = E[:, j].copy()
                for c in cols:
                    e = e - c * np.vdot(c, e)
                nrm = np.linalg.norm(e)
                if nrm > DEPENDENCE_TOLERANCE:
                    cols.append(e / nrm)
            cols = cols[:cap - m]
            k = len(cols)
            if k:
                E = np.stack(cols, axis=1)
                V[:, m:m + k] = E
                S[:m + k, m:m + k] = V[:, :m + k].conj().T @ E
                S[m:m + k, :m + k] = S[:m + k, m:m + k].conj().T
                if not _chol_extend(S, L, m, m + k):
                    raise ValueError("reference overlap remains dependent after repair")
        old = w[:n].copy()
        if k > 0:
            HE = apply(V[:, m:m + k])
            sol.h_columns += k
            HV[:, m:m + k] = HE
            Hr[:m + k, m:m + k] = V[:, :m + k].conj().T @ HE
            Hr[m:m + k, :m + k] = Hr[:m + k, m:m + k].conj().T
            m += k
            w, C = _eigen(Hr, L, m)
        change = np.abs(w[:n] - old)
        sol.ritz_changes.append(change)
        conv = np.array([change[i] < opts.band_threshold(i) for i in range(n)])
        active = [i for i in range(n) if not conv[i]]
        sol.iterations = step + 1
        if not active or sol.iterations == opts.max_iterations:
            break
        if m + len(active) > cap:
            contract(m)
    sol.eigenvalues = w[:n].copy()
    sol.eigenvectors = V[:, :m] @ C[:, :n]
    sol.hx = HV[:, :m] @ C[:, :n]
    sol.converged = conv
    return sol


def dct_fixture(n: int, cluster: bool) -> np.ndarray:
    """The reference's dense Davidson fixture, crates/dft-solvers/tests/ref_davidson.rs:
    55-86: H = Q diag(vals) Q^T in the orthogonal DCT basis; with `cluster`, two
    degenerate pairs (0.3, 0.5), one ending at the occupied edge."""
    i = np.arange(n)
    if cluster:
        vals = np.array([0.3 if k in (2, 3) else 0.5 if k in (4, 5) else 0.1 * k for k in range(n)])
    else:
        vals = 0.2 * i
    q = np.empty((n, n))
    for k in range(n):
        q[:, k] = 1.0 / math.sqrt(n) if k == 0 else math.sqrt(2.0 / n) * np.cos(math.pi * (i + 0.5) * k / n)
    return (q * vals[None, :]) @ q.T


def dct_start(n: int, b: int) -> np.ndarray:
    """ref_davidson.rs:87-98: identity columns plus 0.03 sin(31 i + 17 j + 3)."""
    i = np.arange(n)[:, None]
    j = np.arange(b)[None, :]
    x = 0.03 * np.sin((i * 31 + j * 17 + 3).astype(np.float64))
    x[np.arange(b), np.arange(b)] = 1.0
    return x


def projector_error(a: np.ndarray, b: np.ndarray, k: int) -> float:
    """max |a_k a_k^H - b_k b_k^H| over the leading k columns (ref_davidson.rs:99-110)."""
    pa = a[:, :k] @ a[:, :k].conj().T
    pb = b[:, :k] @ b[:, :k].conj().T
    return float(np.max(np.abs(pa - pb)))
