"""Shared builders for the parity tests: one workload's operator inputs and the
oracle's answer on the same inputs."""
from __future__ import annotations

import numpy as np

from baandi_b200 import operands as O
from oracle import oracle as OR
from oracle import setup_ref as S


def oracle_inputs(w, k):
    """Operands of the oracle for workload w at k (oracle setup, independent of the product)."""
    cell = S.Cell(w.rows)
    b = S.basis_at_k(cell, w.ecut_ha, k)
    species = []
    for s in w.species:
        p = s.pseudo
        ps = S.Pseudo(p.z, p.r, p.rab, p.local, [S.Projector(l, u) for l, u in zip(p.l, p.beta)], p.dij)
        species.append(S.Species(ps, s.positions))
    nl = S.nonlocal_table(b, cell.volume, species)
    return cell, b, nl


def oracle_apply(w, k, dims, vgrid, x, gamma_real=False):
    cell, b, nl = oracle_inputs(w, k)
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    if not gamma_real:
        return OR.apply_complex(dims, idx, vgrid, 0.5 * b.kpg2, nl, x)
    plus, minus, _ = S.half_sphere(b)
    porc = S.orc_projectors(plus, nl.table)
    korc = S.orc_kinetic(plus, b.kpg2)
    return OR.apply_gamma(dims, idx, plus, minus, vgrid, korc, porc, nl, x)


def rel_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def colwise_rel(a, b):
    num = np.linalg.norm(a - b, axis=0)
    den = np.maximum(np.linalg.norm(b, axis=0), 1e-300)
    return float(np.max(num / den))
