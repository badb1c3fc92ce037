"""Oracle (test infrastructure only): FP64 numpy restatement of the learned
preconditioner's network, training samples, loss and gradient.

The reference has no learned preconditioner (its Preconditioner seam,
crates/dft-solvers/src/lib.rs:83-102, takes any correction; TPA is lib.rs:176-207), so
this restates the library's own specification of the learned form rather than reference
code: parity is pinned by finite differences of this restatement and by the identity
"zero output layer = TPA", not against the reference.

Only tests/, the smoke check and bench.py's cpu_baseline leg import this module.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID = 5, 64
OW1 = 0
OB1 = OW1 + N_HID * N_IN
OW2 = OB1 + N_HID
OB2 = OW2 + N_HID * N_HID
OW3 = OB2 + N_HID
OB3 = OW3 + N_HID
NPARAMS = OB3 + 1
CLAMP = 3.0
C0 = 0.7978845608028654  # sqrt(2 / pi)


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OW1:OB1].reshape(N_HID, N_IN), p[OB1:OW2], p[OW2:OB2].reshape(N_HID, N_HID), p[OB2:OW3],
            p[OW3:OB3], p[OB3])


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C0 * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    th = np.tanh(C0 * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * C0 * (1.0 + 3 * 0.044715 * x * x)


def tpa_weight(t, s):
    """TPA factor (crates/dft-solvers/src/lib.rs:176-206), both branches of the device form."""
    t = np.asarray(t, np.float64)
    x = t / s
    p1 = 27.0 + x * (18.0 + x * (12.0 + x * 8.0))
    lo = p1 / (p1 + 16.0 * x ** 4)
    with np.errstate(divide="ignore", invalid="ignore"):
        y = s / t
        p2 = y * (8.0 + y * (12.0 + y * (18.0 + y * 27.0)))
        hi = p2 / (p2 + 16.0)
    return np.where(x <= 1.0, lo, hi)


def features(t, s, lam, rho):
    t = np.asarray(t, np.float64)
    rho = np.asarray(rho, np.float64)
    return np.stack([np.log(np.maximum(t / s, 1e-4)), np.log(t + 0.05), np.full_like(t, np.log(s)),
                     np.full_like(t, lam), np.log(np.clip(rho, 1e-6, 1e6))], axis=1)


def samples(x, hx, e, kin, lam):
    """Samples of one Davidson state (rows x cols): feats, base, a, z, col, ecol."""
    feats, base, a, z, col = [], [], [], [], []
    ecol = []
    for j in range(x.shape[1]):
        w = np.abs(x[:, j]) ** 2
        s = max(np.sum(w * kin) / np.sum(w), 0.1)
        r = hx[:, j] - lam[j] * x[:, j]
        ra = np.abs(r) ** 2
        rms = np.sqrt(np.sum(ra) / len(r))
        feats.append(features(kin, s, lam[j], np.sqrt(ra) / rms if rms > 0 else np.ones_like(ra)))
        base.append(-tpa_weight(kin, s))
        a.append(ra)
        z.append(np.conj(r) * e[:, j])
        col.append(np.full(len(r), j))
        ecol.append(np.sum(np.abs(e[:, j]) ** 2))
    return (np.concatenate(feats), np.concatenate(base), np.concatenate(a), np.concatenate(z), np.concatenate(col),
            np.asarray(ecol))


def forward(p, f):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    pre1 = f @ w1.T + b1
    h1 = gelu(pre1)
    pre2 = h1 @ w2.T + b2
    h2 = gelu(pre2)
    return h2 @ w3 + b3, (pre1, h1, pre2, h2)


def loss_grad(p, feats, base, a, z, col, ecol):
    """Loss (mean over columns of 1 - |A|^2 / (B E)) and its gradient in p."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    m, (pre1, h1, pre2, h2) = forward(p, feats)
    inside = np.abs(m) < CLAMP
    pv = base * np.exp(np.clip(m, -CLAMP, CLAMP))
    nc = len(ecol)
    A = np.zeros(nc, np.complex128)
    B = np.zeros(nc)
    np.add.at(A, col, pv * z)
    np.add.at(B, col, pv * pv * a)
    ok = (B > 0) & (ecol > 0)
    loss = np.sum(np.where(ok, 1.0 - np.abs(A) ** 2 / np.where(ok, B * ecol, 1.0), 0.0)) / nc
    den = np.where(ok, B * ecol * nc, 1.0)
    cA = np.where(ok, 2.0 * A / den, 0.0)
    cB = np.where(ok, 2.0 * np.abs(A) ** 2 / (np.where(ok, B, 1.0) * den), 0.0)
    dp = -np.real(np.conj(cA[col]) * z) + cB[col] * pv * a
    dm = np.where(inside, dp * pv, 0.0)
    g = np.zeros(NPARAMS)
    g[OW3:OB3] = dm @ h2
    g[OB3] = dm.sum()
    d2 = dm[:, None] * w3[None, :] * gelu_grad(pre2)
    g[OW2:OB2] = (d2.T @ h1).ravel()
    g[OB2:OW3] = d2.sum(0)
    d1 = (d2 @ w2) * gelu_grad(pre1)
    g[OW1:OB1] = (d1.T @ feats).ravel()
    g[OB1:OW2] = d1.sum(0)
    return loss, g
